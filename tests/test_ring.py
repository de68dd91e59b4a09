"""Station data rings, CPU side (gx_ring_* on a host-only handle): the ring
geometry against the reference DataStream's own (DataStream::initialise and
updateConfig, datastream.cpp:116-230, 733-763; VDIFDataStream::updateConfig,
vdiffile.cpp:475-493), and the host form of the segment walk against
DataStream / VDIFDataStream::calculateControlParams (datastream.cpp:368-627,
vdiffile.cpp:348-470) of the compiled reference, bit for bit: every control
word of a valid subint, the scan and seconds words of an invalid one, and the
send start.  Segment tables come from the reference's own VDIFDataStream::
dataRead over synthetic VDIF, and from seeded made-up tables with partly
filled segments, gaps, backward time jumps and unread segments."""
import os

import numpy as np
import pytest

from difx_b200 import synth
from difx_b200.jobfiles import Subband, write_job
from oracle import pyoracle
from tests import jobs
from tests import vdif_streams as vs

needs_ref = pytest.mark.skipif(not pyoracle.reference_available(), reason="reference harness not built")

INVALID = -99999999
GEOM = ("bufferbytes", "readbytes", "numsegments", "overflowbytes", "sendbytes", "blockspersend", "controllength",
        "bytespersamplenum", "bytespersampledenom", "bytesbetweenintegerns", "nsinc", "framegranularity",
        "framespersecond")


def _spec(name):
    sb2 = [Subband(8400.0 + 16 * i, 16.0, "U", 128) for i in range(2)]
    if name == "vdif2bit":
        return jobs.spec_c1(name="rg_v2", nstations=3, subbands=sb2, seed=81)
    if name == "mux4":
        return jobs.spec_c1(name="rg_m4", nstations=3, subbands=sb2, mux_threads=4, seed=82)
    if name == "cplx8":
        return jobs.spec_cplx8(name="rg_c8", seed=83)
    if name == "lsb":
        return jobs.spec_lsb(name="rg_l", seed=84)
    if name == "vdif1bit":
        return jobs.spec_c1(name="rg_v1", nstations=3, subbands=sb2, nbits=1, seed=85)
    raise ValueError(name)


def raw_stream(spec, station, nframes, seed, invalid_frac=0.02, perturb=None):
    """Raw frames of one station from the scan start: the job's own VDIF for a
    single-thread station, seeded single-thread frames of every thread (with
    the perturbations asked for) for an interlaced one."""
    if spec.mux_threads <= 0:
        return synth.make_station_stream(spec, station, 0, nframes, seed=seed, invalid_frac=invalid_frac).data.tobytes()
    mt = spec.mux_threads
    fb = spec.payload_bytes // mt + 32
    fps = int(round(spec.frames_per_second))
    return vs.stream(list(range(mt)), nframes, fb, fps, spec.nbits, seed=seed * 7 + station,
                     start_sec=spec.start_seconds, start_frame=0, cplx=spec.is_complex, **(perturb or {}))


def _open(name):
    from difx_b200.gxcorr import Correlator, Ring
    spec = _spec(name)
    paths = write_job(spec, os.path.join(jobs._TMP, "ring_" + name))
    c = Correlator.from_input(paths["input"], device=-1)
    return spec, paths, c, Ring(c)


def same_control(ref_cw, my_cw, ref_start, my_start):
    if ref_cw[0] != my_cw[0] or ref_cw[1] != my_cw[1]:
        return False
    if ref_cw[1] == INVALID:
        return True
    return np.array_equal(ref_cw, my_cw) and ref_start == my_start


@needs_ref
@pytest.mark.parametrize("name", ["vdif2bit", "mux4", "cplx8", "lsb", "vdif1bit"])
def test_ring_geometry_matches_reference_datastream(name):
    spec, paths, c, r = _open(name)
    ref = pyoracle.Reference(paths["input"])
    try:
        for s in range(spec.nstations):
            raw = raw_stream(spec, s, 8, seed=1)
            rd = pyoracle.RefDataStream(ref, s, raw)
            g = r.geometry(s)
            mine = {k: getattr(g, k) for k in GEOM}
            want = {k: rd.geometry[k] for k in GEOM}
            assert mine == want, (name, s, {k: (mine[k], want[k]) for k in GEOM if mine[k] != want[k]})
            assert g.sampletimens == rd.geometry["sampletimens"]
            rd.close()
    finally:
        r.close()
        c.close()
        ref.close()


@needs_ref
@pytest.mark.parametrize("name", ["vdif2bit", "mux4"])
def test_host_walk_matches_reference_on_read_segments(name):
    """The reference's dataRead fills the segments of one station; the same
    segment descriptions go into the ring; then every subint of the data span,
    from the scan start (where the first FFT blocks precede the data), gets
    the same control words and send start from both walks."""
    spec, paths, c, r = _open(name)
    ref = pyoracle.Reference(paths["input"])
    try:
        s = 1
        g = r.geometry(s)
        nfr = int(3.3 * g.readbytes / (spec.payload_bytes + 32)) + 8
        raw = raw_stream(spec, s, nfr, seed=3, perturb=dict(invalid_frac=0.03, drop_frac=0.01))
        rd = pyoracle.RefDataStream(ref, s, raw)
        nread = 0
        for seg in range(3):
            out = rd.read(seg)
            assert out is not None
            r.set_segment(s, seg, (*out[1], 0))
            nread += 1
        span_ns = nread * g.nsinc
        nsub = int((span_ns - 2 * spec.subint_ns) // spec.subint_ns)
        assert nsub >= 8
        invalid = 0
        for k in range(nsub):
            t = k * spec.subint_ns
            sec, ns = t // 10**9, t % 10**9
            cw, sp, _, _ = rd.control(0, sec, ns)
            mw, msp, exhausted = r.control_host(s, 0, sec, ns)
            assert not exhausted
            assert same_control(cw, mw, sp, msp), (name, k, cw[:6], mw[:6], sp, msp)
            invalid += cw[1] == INVALID
        assert invalid < nsub
        rd.close()
    finally:
        r.close()
        c.close()
        ref.close()


@needs_ref
@pytest.mark.parametrize("seed", [1, 2, 3, 4, 5, 6])
def test_host_walk_matches_reference_on_made_up_segments(seed):
    """Seeded segment tables (full, partly filled, empty and unread segments;
    gaps and backward jumps between them; the last one an end marker past the
    data, as the reference's reader leaves after the last file,
    datastream.cpp:940-945) and subints in time order across them."""
    spec, paths, c, r = _open("vdif2bit")
    ref = pyoracle.Reference(paths["input"])
    rng = np.random.default_rng(seed)
    try:
        s = 0
        g = r.geometry(s)
        rd = pyoracle.RefDataStream(ref, s, raw_stream(spec, s, 8, seed=1))
        nseg = g.numsegments
        t = int(rng.integers(0, 3)) * 1_000_000
        table = []
        for k in range(nseg - 1):
            kind = rng.random()
            valid = g.readbytes
            if kind < 0.25:
                valid = int(rng.integers(0, g.readbytes // 8)) * 8
            readto = 0 if rng.random() < 0.05 else 1
            table.append((0, t // 10**9, t % 10**9, valid, readto))
            step = g.nsinc
            j = rng.random()
            if j < 0.15:
                step += int(rng.integers(1, 40)) * 1_000_000          # a gap
            elif j < 0.22:
                step = -int(rng.integers(1, 20)) * 1_000_000          # a backward jump
            t = max(0, t + step)
        table.append((0, 2, 0, g.readbytes, 1))                        # end marker: past the data
        for k, seg in enumerate(table):
            rd.set_segment(k, seg)
            r.set_segment(s, k, (*seg, 0))
        end_ns = max(x[1] * 10**9 + x[2] for x in table[:-1]) + g.nsinc
        times = np.sort(rng.integers(0, end_ns, 40))
        for t in times:
            t = int(t)
            sec, ns = t // 10**9, t % 10**9
            cw, sp, _, _ = rd.control(0, sec, ns)
            mw, msp, _ = r.control_host(s, 0, sec, ns)
            assert same_control(cw, mw, sp, msp), (seed, t, cw[:6], mw[:6], sp, msp)
        rd.close()
    finally:
        r.close()
        c.close()
        ref.close()


def test_ring_needs_a_model():
    from difx_b200 import capi
    from difx_b200.gxcorr import Correlator, GxError, Ring
    c = Correlator.from_desc(capi.job_desc_from_spec(_spec("vdif2bit")), device=-1)
    with pytest.raises(GxError) as ei:
        Ring(c)
    assert ei.value.status == 8
    c.close()
