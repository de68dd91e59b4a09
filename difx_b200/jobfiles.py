"""Writers for DiFX job setup files: ``.input``, ``.calc``, ``.im``, ``.threads``.

The layout follows what the reference correlator's parsers read:

* ``.input``  -- ``Configuration::parseConfiguration`` and its table readers
  (mpifxcorr/src/configuration.cpp:198-345, processCommon 1271, processConfig
  1315, processRuleTable 1891, processFreqTable 1970, processTelescopeTable
  2025, processDatastreamTable 1397, processBaselineTable 1033,
  processDataTable 1956).  Keys are padded to column 20
  (``Configuration::DEFAULT_KEY_LENGTH``, configuration.h:1118).
* ``.calc``   -- ``Model::readInfoData`` ... ``readSpacecraftData``
  (mpifxcorr/src/model.cpp:362-590).
* ``.im``     -- ``Model::readPolynomialSamples`` (model.cpp:596-837).
* ``.threads`` -- read at the end of processDatastreamTable
  (configuration.cpp:1857-1883).

A :class:`JobSpec` describes one single-scan, single-configuration job in
which every station records the same set of subbands (the shape of all the
correlation jobs this package targets).  Delay models are seeded quadratics
written as order-5 ``.im`` polynomials; station clocks are written into the
telescope table.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Sequence, Tuple

import numpy as np

VDIF_HEADER_BYTES = 32


def _kv(key: str, val) -> str:
    k = key + ":"
    return f"{k:<20}{val}\n"


@dataclasses.dataclass
class Subband:
    freq_mhz: float          # band edge (LO) frequency, MHz
    bw_mhz: float
    sideband: str = "U"      # 'U' or 'L'
    nchan: int = 128


@dataclasses.dataclass
class JobSpec:
    name: str = "gxjob"
    nstations: int = 4
    subbands: Sequence[Subband] = ()
    pols: Tuple[str, ...] = ("R", "L")
    nbits: int = 2
    sampling: str = "REAL"            # REAL or COMPLEX
    payload_bytes: int = 8000         # VDIF payload bytes per frame
    start_mjd: int = 57000
    start_seconds: int = 3600         # seconds of day (integer)
    execute_seconds: int = 2
    int_time: float = 0.5
    subint_ns: int = 8_000_000
    guard_ns: int = 0
    fringe_rot_order: int = 1
    array_stride: int = 0             # 0: auto (calcstridelength)
    xmac_stride: int = 0              # 0: auto (calcgoodxmacstridelength)
    num_buffered_ffts: int = 10
    write_autocorrs: bool = True
    full_pol: bool = True             # cross-hand products on every baseline
    seed: int = 1
    max_delay_us: float = 20000.0     # |tau| bound for the seeded delay models
    max_rate_us_per_s: float = 3.0    # |dtau/dt| bound
    max_accel_us_per_s2: float = 1e-4
    clock_us: Sequence[float] = ()    # per-station clock offset (us); default 0
    clock_rate: Sequence[float] = ()  # per-station clock rate (us/s); default 0
    uvshift_interval_ns: int = 2_000_000_000
    ac_avg_interval_ns: int = 2_000_000_000
    chans_to_avg: int = 1             # CHANS TO AVG of every freq (output channels = nchan / this)
    pcal_interval_mhz: int = 0        # PHASE CAL INT (MHZ) of every datastream (0: no phase-cal)
    mux_threads: int = 0              # >0: INTERLACEDVDIF of this many threads, muxed frames with EDV4 headers
    tsys: float = 0.0                 # TSYS of every datastream (> 0: a-priori amplitude calibration)
    edv4_partial_frac: float = 0.0    # fraction of muxed frames whose EDV4 validity mask lacks some threads
    poly_interval_s: int = 120
    station_names: Sequence[str] = ()
    data_files: Sequence[str] = ()
    # per station, the indices into `subbands` it records (default: all of
    # them); every station records the same number
    station_subbands: Sequence[Sequence[int]] = ()
    # zoom freqs (freq-table entries after the subbands): each station
    # correlates each one that lies within one of its recorded subbands, in
    # every polarisation
    zooms: Sequence[Subband] = ()
    zoom_only: bool = False           # baselines correlate the zoom freqs only
    zoom_pols: Tuple[str, ...] = ()   # polarisations of the zoom bands (default: pols)
    # phase centres: with more than one, source 0 is the (uncorrelated)
    # pointing centre and sources 1..n the phase centres, each with a seeded
    # delay offset of up to max_pc_offset_us and rate of up to
    # max_pc_rate_us_per_s relative to the pointing centre
    phase_centres: int = 1
    max_pc_offset_us: float = 0.02
    max_pc_rate_us_per_s: float = 0.002
    # pulsar binning: bins (0: none) of equal phase width, their weights
    # (default 1), scrunched output, and a synthetic pulsar's polyco
    pulsar_bins: int = 0
    pulsar_bin_weights: Sequence[float] = ()
    pulsar_scrunch: bool = False
    pulsar_f0: float = 503.7          # Hz
    pulsar_dm: float = 500.0          # pc cm^-3

    # ------------------------------------------------------------ derived
    def station_sb(self, station: int) -> List[int]:
        """Indices into `subbands` of the subbands a station records."""
        if self.station_subbands:
            return list(self.station_subbands[station])
        return list(range(len(self.subbands)))

    def station_zooms(self, station: int) -> List[Tuple[int, int]]:
        """(zoom index, local recorded freq of its parent) of each zoom freq the
        station correlates: the last recorded subband containing it, as the
        reference's search leaves it (configuration.cpp:1718-1737)."""
        out = []
        sbs = self.station_sb(station)
        for k, z in enumerate(self.zooms):
            zlo = z.freq_mhz - (z.bw_mhz if z.sideband == "L" else 0.0)
            parent = -1
            for j, i in enumerate(sbs):
                p = self.subbands[i]
                plo = p.freq_mhz - (p.bw_mhz if p.sideband == "L" else 0.0)
                if zlo >= plo and zlo + z.bw_mhz <= plo + p.bw_mhz:
                    parent = j
            if parent >= 0:
                out.append((k, parent))
        return out

    @property
    def nbands(self) -> int:
        """Recorded bands per station."""
        return len(self.station_sb(0)) * len(self.pols)

    @property
    def zpols(self) -> Tuple[str, ...]:
        return tuple(self.zoom_pols) if self.zoom_pols else tuple(self.pols)

    @property
    def is_complex(self) -> bool:
        return self.sampling.upper() != "REAL"

    @property
    def bw_mhz(self) -> float:
        return self.subbands[0].bw_mhz

    @property
    def nchan(self) -> int:
        return self.subbands[0].nchan

    @property
    def fftchannels(self) -> int:
        return self.nchan if self.is_complex else 2 * self.nchan

    @property
    def samples_per_second(self) -> float:
        """Time samples per second per band (real or complex)."""
        return self.bw_mhz * 1e6 * (1.0 if self.is_complex else 2.0)

    @property
    def bits_per_timesample(self) -> int:
        return self.nbands * self.nbits * (2 if self.is_complex else 1)

    @property
    def frame_samples(self) -> int:
        return self.payload_bytes * 8 // self.bits_per_timesample

    @property
    def framebytes(self) -> int:
        return self.payload_bytes + VDIF_HEADER_BYTES

    @property
    def frames_per_second(self) -> float:
        return self.samples_per_second / self.frame_samples

    @property
    def blocks_per_send(self) -> int:
        ffttime_ns = 1000.0 * self.nchan / self.bw_mhz
        b = self.subint_ns / ffttime_ns
        if abs(b - round(b)) > 1e-9:
            raise ValueError("subint is not a whole number of FFT blocks")
        return int(round(b))

    def names(self) -> List[str]:
        if self.station_names:
            return list(self.station_names)
        return [_stname(i) for i in range(self.nstations)]

    def validate(self):
        if not self.subbands:
            raise ValueError("no subbands")
        for sb in self.subbands:
            if sb.bw_mhz != self.bw_mhz or sb.nchan != self.nchan:
                raise ValueError("all subbands must share bandwidth and channel count")
        if self.station_subbands and (len(self.station_subbands) != self.nstations or
                                      len({len(x) for x in self.station_subbands}) != 1):
            raise ValueError("every station must record the same number of subbands")
        for z in self.zooms:
            if abs(z.bw_mhz / z.nchan - self.bw_mhz / self.nchan) > 1e-9:
                raise ValueError("a zoom freq's channel width must equal the subbands'")
        if self.bits_per_timesample % 8 != 0 and 8 % self.bits_per_timesample != 0:
            raise ValueError("a time sample of all bands must fill whole bytes or divide a byte")
        if (self.payload_bytes * 8) % self.bits_per_timesample != 0:
            raise ValueError("payload is not a whole number of time samples")
        fps = self.frames_per_second
        if abs(fps - round(fps)) > 1e-9:
            raise ValueError("frames per second must be an integer")
        if self.mux_threads > 0 and (self.payload_bytes % (8 * self.mux_threads) != 0 or
                                     self.mux_threads > 64):
            raise ValueError("each thread's payload must be a whole number of 8-byte words (<= 64 threads)")
        _ = self.blocks_per_send

    # ------------------------------------------------------------ model
    def delay_models(self) -> np.ndarray:
        """Seeded quadratic geometric delays, us: tau(t)=c0+c1 t+c2 t^2 (t s from job start).

        Station 0 is the reference (zero delay is not required; every
        station gets its own seeded model)."""
        rng = np.random.default_rng(self.seed * 7919 + 17)
        span = float(self.execute_seconds)
        c = np.zeros((self.nstations, 3))
        for s in range(self.nstations):
            c2 = rng.uniform(-1, 1) * self.max_accel_us_per_s2
            c1 = rng.uniform(-1, 1) * (self.max_rate_us_per_s - 2 * abs(c2) * span)
            c0 = rng.uniform(-1, 1) * (self.max_delay_us - abs(c1) * span - abs(c2) * span * span)
            c[s] = (c0, c1, c2)
        return c


def phase_centre_offsets(spec: JobSpec) -> np.ndarray:
    """Per phase centre and station (offset us, rate us/s) added to the
    pointing centre's delay model."""
    rng = np.random.default_rng(spec.seed * 31337 + 5)
    out = np.zeros((max(1, spec.phase_centres), spec.nstations, 2))
    if spec.phase_centres > 1:
        out[..., 0] = rng.uniform(-1, 1, out.shape[:2]) * spec.max_pc_offset_us
        out[..., 1] = rng.uniform(-1, 1, out.shape[:2]) * spec.max_pc_rate_us_per_s
    return out


def uvw_poly_rows(spec: JobSpec, nsamp: int) -> np.ndarray:
    """Seeded (u, v, w) polynomials per model sample and station, metres, order 5 in
    seconds from the sample start: a position of up to 6000 km drifting at up to
    450 m/s with a small quadratic term.  Shape [nsamp, nstations, 3, 6]."""
    rng = np.random.default_rng(spec.seed * 104729 + 3)
    out = np.zeros((nsamp, spec.nstations, 3, 6))
    for s in range(spec.nstations):
        p0 = rng.uniform(-6.0e6, 6.0e6, 3)
        rate = rng.uniform(-450.0, 450.0, 3)
        acc = rng.uniform(-0.03, 0.03, 3)
        for k in range(nsamp):
            t0 = k * spec.poly_interval_s
            out[k, s, :, 0] = p0 + rate * t0 + acc * t0 * t0
            out[k, s, :, 1] = rate + 2 * acc * t0
            out[k, s, :, 2] = acc
    return out


def _stname(i: int) -> str:
    a = "ABCDEFGHIJKLMNOPQRSTUVWXYZ"
    return a[(i // 26) % 26] + a[i % 26]


def _mjd_to_ymd(mjd: int):
    # Fliegel & Van Flandern via JD
    jd = mjd + 2400001
    l = jd + 68569
    n = 4 * l // 146097
    l = l - (146097 * n + 3) // 4
    i = 4000 * (l + 1) // 1461001
    l = l - 1461 * i // 4 + 31
    j = 80 * l // 2447
    day = l - 2447 * j // 80
    l = j // 11
    month = j + 2 - 12 * l
    year = 100 * (n - 49) + i + l
    return year, month, day


def delay_poly_rows(spec: JobSpec, coeffs: np.ndarray, nsamples: int) -> np.ndarray:
    """Per-interval order-5 .im polynomial rows [sample][station][6] (us, us/s^n).

    Interval k starts at t_k = k*poly_interval_s seconds after job start and its
    polynomial is in dt = t - t_k, so tau(t_k+dt) = tau(t_k) + tau'(t_k) dt + c2 dt^2."""
    rows = np.zeros((nsamples, spec.nstations, 6))
    for k in range(nsamples):
        tk = float(k * spec.poly_interval_s)
        for s in range(spec.nstations):
            c0, c1, c2 = coeffs[s]
            rows[k, s, 0] = c0 + c1 * tk + c2 * tk * tk
            rows[k, s, 1] = c1 + 2 * c2 * tk
            rows[k, s, 2] = c2
    return rows


def baseline_plan(spec: JobSpec) -> List[Tuple[int, int, List[Tuple[int, List[Tuple[int, int]]]]]]:
    """The baseline table: (datastream A, datastream B, [(freq-table index,
    [(band A, band B) per polarisation product])]).  Freqs are the recorded
    subbands both stations record (unless zoom_only), then the zoom freqs both
    correlate; band indices count the recorded bands, then the zoom bands, as
    the reference does (configuration.cpp:1095-1115)."""
    npol = len(spec.pols)
    nsb = len(spec.subbands)
    prods = []
    for p1 in range(npol):
        for p2 in range(npol):
            if p1 == p2 or spec.full_pol:
                prods.append((p1, p2))
    # DiFX order: parallel hands first, then cross hands (RR, LL, RL, LR)
    prods.sort(key=lambda t: (t[0] != t[1], t))
    out = []
    for a in range(spec.nstations):
        for b in range(a + 1, spec.nstations):
            sa, sb_ = spec.station_sb(a), spec.station_sb(b)
            za = [k for k, _ in spec.station_zooms(a)]
            zb = [k for k, _ in spec.station_zooms(b)]
            freqs = []
            if not spec.zoom_only:
                for i in range(nsb):
                    if i in sa and i in sb_:
                        freqs.append((i, [(sa.index(i) * npol + p1, sb_.index(i) * npol + p2) for p1, p2 in prods]))
            zp = spec.zpols
            nzp = len(zp)
            zprods = []
            for p1 in range(nzp):
                for p2 in range(nzp):
                    if p1 == p2 or spec.full_pol:
                        zprods.append((p1, p2))
            zprods.sort(key=lambda t: (t[0] != t[1], t))
            for k in range(len(spec.zooms)):
                if k in za and k in zb:
                    freqs.append((nsb + k, [(spec.nbands + za.index(k) * nzp + p1, spec.nbands + zb.index(k) * nzp + p2)
                                            for p1, p2 in zprods]))
            out.append((a, b, freqs))
    return out


def _fortran_d(x: float) -> str:
    return f"{x:25.17E}".replace("E", "D")


def write_polyco(spec: JobSpec, path: str) -> None:
    """A one-entry TEMPO-style polyco (the layout Configuration counts entries
    by and Polyco::loadPolycoFile reads, polyco.cpp:399-524): a 2-hour span
    centred on the job, the phase polynomial in minutes from that centre."""
    mjd_mid = spec.start_mjd + (spec.start_seconds + spec.execute_seconds / 2.0) / 86400.0
    frac = mjd_mid - int(mjd_mid)
    hh = int(frac * 24)
    mm = int((frac * 24 - hh) * 60)
    ss = ((frac * 24 - hh) * 60 - mm) * 60
    coeffs = [0.137, 2.0e-3, 1.5e-5, -2.0e-8] + [0.0] * 8
    utc = f"{hh:02d}{mm:02d}{ss:05.2f}"
    l1 = f"{'J0000+00':<10s}{'01-JAN-15':>10s}{utc:>12s}{mjd_mid:20.11f}{spec.pulsar_dm:21.6f}{0.0:7.3f}{-6.0:7.3f}"
    l2 = f"{0.25:20.6f}{spec.pulsar_f0:18.12f}{'    7':>5s}{120:5d}{len(coeffs):5d}{8400.0:10.3f}"
    lines = [l1, l2]
    for k in range(0, len(coeffs), 3):
        lines.append("".join(_fortran_d(c) for c in coeffs[k:k + 3]))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_job(spec: JobSpec, outdir: str) -> dict:
    """Write ``<name>.input/.calc/.im/.threads/.flag`` into outdir; return their paths."""
    spec.validate()
    os.makedirs(outdir, exist_ok=True)
    base = os.path.join(outdir, spec.name)
    paths = {k: base + "." + k for k in ("input", "calc", "im", "threads", "flag")}
    if spec.pulsar_bins > 0:
        paths["binconfig"] = base + ".binconfig"
        paths["polyco"] = base + ".polyco"
        write_polyco(spec, paths["polyco"])
        B = [_kv("NUM POLYCO FILES", 1), _kv("POLYCO FILE 0", paths["polyco"]),
             _kv("NUM PULSAR BINS", spec.pulsar_bins), _kv("SCRUNCH OUTPUT", "TRUE" if spec.pulsar_scrunch else "FALSE")]
        for k in range(spec.pulsar_bins):
            w = spec.pulsar_bin_weights[k] if k < len(spec.pulsar_bin_weights) else 1.0
            B.append(_kv(f"BIN PHASE END {k}", f"{(k + 1) / spec.pulsar_bins:.6f}"))
            B.append(_kv(f"BIN WEIGHT {k}", f"{w:.6f}"))
        with open(paths["binconfig"], "w") as f:
            f.write("".join(B))
    names = spec.names()
    nst = spec.nstations
    nsb = len(spec.subbands)
    npol = len(spec.pols)

    # ---------------------------------------------------------------- .threads
    with open(paths["threads"], "w") as f:
        f.write(_kv("NUMBER OF CORES", 1))
        f.write("1\n")
    with open(paths["flag"], "w") as f:
        f.write("0\n")

    # ---------------------------------------------------------------- .input
    L = []
    L.append("# COMMON SETTINGS ##!\n")
    L.append(_kv("CALC FILENAME", paths["calc"]))
    L.append(_kv("CORE CONF FILENAME", paths["threads"]))
    L.append(_kv("EXECUTE TIME (SEC)", spec.execute_seconds))
    L.append(_kv("START MJD", spec.start_mjd))
    L.append(_kv("START SECONDS", spec.start_seconds))
    L.append(_kv("ACTIVE DATASTREAMS", nst))
    nbl = nst * (nst - 1) // 2
    L.append(_kv("ACTIVE BASELINES", nbl))
    L.append(_kv("VIS BUFFER LENGTH", 80))
    L.append(_kv("OUTPUT FORMAT", "SWIN"))
    L.append(_kv("OUTPUT FILENAME", base + ".difx"))
    L.append("\n# CONFIGURATIONS ###!\n")
    L.append(_kv("NUM CONFIGURATIONS", 1))
    L.append(_kv("CONFIG NAME", "gxcfg"))
    L.append(_kv("INT TIME (SEC)", f"{spec.int_time:.6f}"))
    L.append(_kv("SUBINT NANOSECONDS", spec.subint_ns))
    L.append(_kv("GUARD NANOSECONDS", spec.guard_ns))
    L.append(_kv("FRINGE ROTN ORDER", spec.fringe_rot_order))
    L.append(_kv("ARRAY STRIDE LENGTH", spec.array_stride))
    L.append(_kv("XMAC STRIDE LENGTH", spec.xmac_stride))
    L.append(_kv("NUM BUFFERED FFTS", spec.num_buffered_ffts))
    L.append(_kv("WRITE AUTOCORRS", "TRUE" if spec.write_autocorrs else "FALSE"))
    if spec.pulsar_bins > 0:
        L.append(_kv("PULSAR BINNING", "TRUE"))
        L.append(_kv("PULSAR CONFIG FILE", paths["binconfig"]))
    else:
        L.append(_kv("PULSAR BINNING", "FALSE"))
    L.append(_kv("PHASED ARRAY", "FALSE"))
    for i in range(nst):
        L.append(_kv(f"DATASTREAM {i} INDEX", i))
    for i in range(nbl):
        L.append(_kv(f"BASELINE {i} INDEX", i))
    L.append("\n# RULES ############!\n")
    L.append(_kv("NUM RULES", 1))
    L.append(_kv("RULE 0 SCAN ID", "SCAN0"))
    L.append(_kv("RULE 0 CONFIG NAME", "gxcfg"))
    L.append("\n# FREQ TABLE #######!\n")
    L.append(_kv("FREQ ENTRIES", nsb + len(spec.zooms)))
    for i, sb in enumerate(list(spec.subbands) + list(spec.zooms)):
        L.append(_kv(f"FREQ (MHZ) {i}", f"{sb.freq_mhz:.11f}"))
        L.append(_kv(f"BW (MHZ) {i}", f"{sb.bw_mhz:.11f}"))
        L.append(_kv(f"SIDEBAND {i}", sb.sideband))
        L.append(_kv(f"NUM CHANNELS {i}", sb.nchan))
        L.append(_kv(f"CHANS TO AVG {i}", spec.chans_to_avg))
        L.append(_kv(f"OVERSAMPLE FAC. {i}", 1))
        L.append(_kv(f"DECIMATION FAC. {i}", 1))
        L.append(_kv(f"PHASE CALS {i} OUT", 0))
    L.append("\n# TELESCOPE TABLE ##!\n")
    L.append(_kv("TELESCOPE ENTRIES", nst))
    for i in range(nst):
        L.append(_kv(f"TELESCOPE NAME {i}", names[i]))
        L.append(_kv(f"CLOCK REF MJD {i}", f"{spec.start_mjd + spec.start_seconds / 86400.0:.10f}"))
        L.append(_kv(f"CLOCK POLY ORDER {i}", 1))
        L.append("@ ***** Clock poly coeff N: has units microsec / sec^N ***** @\n")
        c0 = spec.clock_us[i] if i < len(spec.clock_us) else 0.0
        c1 = spec.clock_rate[i] if i < len(spec.clock_rate) else 0.0
        L.append(_kv(f"CLOCK COEFF {i}/0", f"{c0:.15e}"))
        L.append(_kv(f"CLOCK COEFF {i}/1", f"{c1:.15e}"))
    L.append("\n# DATASTREAM TABLE #!\n")
    L.append(_kv("DATASTREAM ENTRIES", nst))
    L.append(_kv("DATA BUFFER FACTOR", 32))
    L.append(_kv("NUM DATA SEGMENTS", 8))
    samp = "REAL" if not spec.is_complex else "COMPLEX"
    for i in range(nst):
        L.append(_kv("TELESCOPE INDEX", i))
        L.append(_kv("TSYS", f"{spec.tsys:.6f}"))
        if spec.mux_threads > 0:
            # per-thread frames before multiplexing; the Core sees spec.framebytes
            L.append(_kv("DATA FORMAT", "INTERLACEDVDIF/" + ":".join(str(t) for t in range(spec.mux_threads))))
            L.append(_kv("QUANTISATION BITS", spec.nbits))
            L.append(_kv("DATA FRAME SIZE", spec.payload_bytes // spec.mux_threads + VDIF_HEADER_BYTES))
        else:
            L.append(_kv("DATA FORMAT", "VDIF"))
            L.append(_kv("QUANTISATION BITS", spec.nbits))
            L.append(_kv("DATA FRAME SIZE", spec.framebytes))
        L.append(_kv("DATA SAMPLING", samp))
        L.append(_kv("DATA SOURCE", "FILE"))
        L.append(_kv("FILTERBANK USED", "FALSE"))
        L.append(_kv("PHASE CAL INT (MHZ)", spec.pcal_interval_mhz))
        sbs = spec.station_sb(i)
        L.append(_kv("NUM RECORDED FREQS", len(sbs)))
        for j, g in enumerate(sbs):
            L.append(_kv(f"REC FREQ INDEX {j}", g))
            L.append(_kv(f"CLK OFFSET {j} (us)", "0.000000"))
            L.append(_kv(f"FREQ OFFSET {j} (Hz)", "0.000000"))
            L.append(_kv(f"NUM REC POLS {j}", npol))
        b = 0
        for j in range(len(sbs)):
            for p in spec.pols:
                L.append(_kv(f"REC BAND {b} POL", p))
                L.append(_kv(f"REC BAND {b} INDEX", j))
                b += 1
        zl = spec.station_zooms(i)
        L.append(_kv("NUM ZOOM FREQS", len(zl)))
        for j, (k, _) in enumerate(zl):
            L.append(_kv(f"ZOOM FREQ INDEX {j}", nsb + k))
            L.append(_kv(f"NUM ZOOM POLS {j}", len(spec.zpols)))
        b = 0
        for j in range(len(zl)):
            for p in spec.zpols:
                L.append(_kv(f"ZOOM BAND {b} POL", p))
                L.append(_kv(f"ZOOM BAND {b} INDEX", j))
                b += 1
    L.append("\n# BASELINE TABLE ###!\n")
    L.append(_kv("BASELINE ENTRIES", nbl))
    for bl, (a, bb, freqs) in enumerate(baseline_plan(spec)):
        L.append(_kv(f"D/STREAM A INDEX {bl}", a))
        L.append(_kv(f"D/STREAM B INDEX {bl}", bb))
        L.append(_kv(f"NUM FREQS {bl}", len(freqs)))
        for j, (f, pairs) in enumerate(freqs):
            L.append(_kv(f"TARGET FREQ {bl}/{j}", f))
            L.append(_kv(f"POL PRODUCTS {bl}/{j}", len(pairs)))
            for k, (b1, b2) in enumerate(pairs):
                L.append(_kv(f"D/STREAM A BAND {k}", b1))
                L.append(_kv(f"D/STREAM B BAND {k}", b2))
    L.append("\n# DATA TABLE #######!\n")
    for i in range(nst):
        L.append(_kv(f"D/STREAM {i} FILES", 1))
        fn = spec.data_files[i] if i < len(spec.data_files) else f"{base}.st{i}.vdif"
        L.append(_kv(f"FILE {i}/0", fn))
    L.append("\n")
    with open(paths["input"], "w") as f:
        f.write("".join(L))

    # ---------------------------------------------------------------- .calc
    y, mo, d = _mjd_to_ymd(spec.start_mjd)
    hh = spec.start_seconds // 3600
    mi = (spec.start_seconds % 3600) // 60
    ss = spec.start_seconds % 60
    start_mjd_f = spec.start_mjd + spec.start_seconds / 86400.0
    stop_mjd_f = start_mjd_f + spec.execute_seconds / 86400.0
    C = []
    C.append(_kv("JOB ID", 1))
    C.append(_kv("JOB START TIME", f"{start_mjd_f:.7f}"))
    C.append(_kv("JOB STOP TIME", f"{stop_mjd_f:.7f}"))
    C.append(_kv("DUTY CYCLE", "1.000"))
    C.append(_kv("OBSCODE", "GXSYN"))
    C.append(_kv("DIFX VERSION", "gxcorr"))
    C.append(_kv("SUBJOB ID", 0))
    C.append(_kv("SUBARRAY ID", 0))
    C.append(_kv("VEX FILE", "none.vex"))
    C.append(_kv("START MJD", f"{start_mjd_f:.7f}"))
    C.append(_kv("START YEAR", y))
    C.append(_kv("START MONTH", mo))
    C.append(_kv("START DAY", d))
    C.append(_kv("START HOUR", hh))
    C.append(_kv("START MINUTE", mi))
    C.append(_kv("START SECOND", ss))
    C.append(_kv("SPECTRAL AVG", 1))
    C.append(_kv("TAPER FUNCTION", "UNIFORM"))
    C.append(_kv("NUM TELESCOPES", nst))
    rng = np.random.default_rng(spec.seed + 101)
    for i in range(nst):
        C.append(_kv(f"TELESCOPE {i} NAME", names[i]))
        C.append(_kv(f"TELESCOPE {i} MOUNT", "AZEL"))
        C.append(_kv(f"TELESCOPE {i} OFFSET (m)", "0.000000"))
        xyz = rng.normal(size=3)
        xyz = 6.371e6 * xyz / np.linalg.norm(xyz)
        C.append(_kv(f"TELESCOPE {i} X (m)", f"{xyz[0]:.6f}"))
        C.append(_kv(f"TELESCOPE {i} Y (m)", f"{xyz[1]:.6f}"))
        C.append(_kv(f"TELESCOPE {i} Z (m)", f"{xyz[2]:.6f}"))
        C.append(_kv(f"TELESCOPE {i} SHELF", "NONE"))
    npc = max(1, spec.phase_centres)
    srcnames = ["SYNTH"] + ([f"PC{j}" for j in range(npc)] if npc > 1 else [])
    C.append(_kv("NUM SOURCES", len(srcnames)))
    for j, nm in enumerate(srcnames):
        C.append(_kv(f"SOURCE {j} NAME", nm))
        C.append(_kv(f"SOURCE {j} RA", f" {1.0 + 1e-5 * j:.16f}"))
        C.append(_kv(f"SOURCE {j} DEC", f" {0.5 + 1e-5 * j:.16f}"))
        C.append(_kv(f"SOURCE {j} CALCODE", " "))
        C.append(_kv(f"SOURCE {j} QUAL", 0))
    C.append(_kv("NUM SCANS", 1))
    C.append(_kv("SCAN 0 IDENTIFIER", "SCAN0"))
    C.append(_kv("SCAN 0 START (S)", 0))
    C.append(_kv("SCAN 0 DUR (S)", spec.execute_seconds))
    C.append(_kv("SCAN 0 OBS MODE NAME", "gxmode"))
    C.append(_kv("SCAN 0 UVSHIFT INTERVAL (NS)", spec.uvshift_interval_ns))
    C.append(_kv("SCAN 0 AC AVG INTERVAL (NS)", spec.ac_avg_interval_ns))
    C.append(_kv("SCAN 0 POINTING SRC", 0))
    C.append(_kv("SCAN 0 NUM PHS CTRS", npc))
    for j in range(npc):
        C.append(_kv(f"SCAN 0 PHS CTR {j}", j + 1 if npc > 1 else 0))
    C.append(_kv("NUM EOPS", 0))
    C.append(_kv("NUM SPACECRAFT", 0))
    C.append(_kv("IM FILENAME", paths["im"]))
    C.append(_kv("FLAG FILENAME", paths["flag"]))
    with open(paths["calc"], "w") as f:
        f.write("".join(C))

    # ---------------------------------------------------------------- .im
    nsamp = int(math.ceil(spec.execute_seconds / spec.poly_interval_s)) + 1
    rows = delay_poly_rows(spec, spec.delay_models(), nsamp)
    I = []
    I.append(_kv("CALC SERVER", "gxsynth"))
    I.append(_kv("CALC PROGRAM", -1))
    I.append(_kv("CALC VERSION", -1))
    I.append(_kv("START YEAR", y))
    I.append(_kv("START MONTH", mo))
    I.append(_kv("START DAY", d))
    I.append(_kv("START HOUR", hh))
    I.append(_kv("START MINUTE", mi))
    I.append(_kv("START SECOND", ss))
    I.append(_kv("POLYNOMIAL ORDER", 5))
    I.append(_kv("INTERVAL (SECS)", spec.poly_interval_s))
    I.append(_kv("ABERRATION CORR", "EXACT"))
    I.append(_kv("NUM TELESCOPES", nst))
    for i in range(nst):
        I.append(_kv(f"TELESCOPE {i} NAME", names[i]))
    I.append(_kv("NUM SCANS", 1))
    I.append(_kv("SCAN 0 POINTING SRC", "SYNTH"))
    I.append(_kv("SCAN 0 NUM PHS CTRS", npc))
    for j in range(npc):
        I.append(_kv(f"SCAN 0 PHS CTR {j} SRC", srcnames[j + 1] if npc > 1 else "SYNTH"))
    I.append(_kv("SCAN 0 NUM POLY", nsamp))
    uvw = uvw_poly_rows(spec, nsamp)
    for k in range(nsamp):
        t = spec.start_seconds + k * spec.poly_interval_s
        I.append(_kv(f"SCAN 0 POLY {k} MJD", spec.start_mjd + t // 86400))
        I.append(_kv(f"SCAN 0 POLY {k} SEC", t % 86400))
        pco = phase_centre_offsets(spec)
        for src in range(npc + 1):
            for s in range(nst):
                row = rows[k, s].copy()
                if npc > 1 and src > 0:   # phase centre src: offset + rate (t from the poly start)
                    row[0] += pco[src - 1, s, 0] + pco[src - 1, s, 1] * k * spec.poly_interval_s
                    row[1] += pco[src - 1, s, 1]
                vals = "\t ".join(f"{v:.16e}" for v in row)
                I.append(_kv(f"SRC {src} ANT {s} DELAY (us)", vals))
                for c, name in enumerate("UVW"):
                    I.append(_kv(f"SRC {src} ANT {s} {name} (m)", "\t ".join(f"{v:.16e}" for v in uvw[k, s, c])))
    with open(paths["im"], "w") as f:
        f.write("".join(I))
    return paths
