"""The C-ABI library loads and exports every entry point include/gxcorr.h
declares; host-only handles work without a GPU; descriptor errors are
reported as status codes, not crashes."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from difx_b200 import capi, gxcorr
from tests import jobs

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "gxcorr.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    # function declarations: a return type at the start of a line, then the name and "("
    return sorted(set(re.findall(r"^\s*(?:gx_status|const\s+char\s*\*)\s*(gx_[a-z_]+)\s*\(", src, re.M)))


def test_header_and_binding_agree():
    decl = declared_functions()
    assert decl, "no declarations parsed"
    assert sorted(gxcorr.EXPORTED_SYMBOLS) == decl


def test_library_exports_every_declared_symbol():
    lib = gxcorr.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name


@pytest.mark.skipif(not os.path.exists("/usr/bin/gcc"), reason="no C compiler")
def test_struct_layout_matches_c_compiler(tmp_path):
    """ctypes mirrors of the ABI structs have the C compiler's sizes and offsets."""
    import subprocess
    structs = {"gx_freq_desc": capi.gx_freq_desc, "gx_station_desc": capi.gx_station_desc,
               "gx_baseline_desc": capi.gx_baseline_desc, "gx_job_desc": capi.gx_job_desc,
               "gx_subint_desc": capi.gx_subint_desc, "gx_layout_info": capi.gx_layout_info,
               "gx_vdifmux_stats": gxcorr.VdifMuxStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for name, cls in structs.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["/usr/bin/gcc", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(l.split() for l in out if l.strip())
    for name, cls in structs.items():
        assert int(got[name]) == C.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(got[f"{name}.{fname}"]) == getattr(cls, fname).offset, (name, fname)


def test_host_only_handle_layout():
    spec = jobs.spec_c1()
    jd = capi.job_desc_from_spec(spec)
    c = gxcorr.Correlator.from_desc(jd, device=-1)
    assert c.info.nchan == spec.nchan
    assert c.info.fftchannels == 2 * spec.nchan
    assert c.info.blocks_per_send == spec.blocks_per_send
    assert c.info.array_stride == 16 and c.info.xmac_stride == 128
    with pytest.raises(gxcorr.GxError) as ei:
        c.subint(capi.SubintDesc(0, 0, 0, 0.0, [0] * 4, [0] * 4, [0] * 4, 3))
    assert ei.value.status == 8   # GX_ERR_STATE: host-only handle
    c.close()


@pytest.mark.parametrize("mutate,status", [
    (lambda d: setattr(d.desc, "fringe_rotation_order", 3), 2),
    (lambda d: setattr(d.desc, "fringe_rotation_order", -1), 2),
    (lambda d: setattr(d.desc, "subint_ns", 8_000_001), 1),
    (lambda d: setattr(d._st[1], "nbits", 8), 2),
])
def test_bad_descriptors_are_rejected(mutate, status):
    jd = capi.job_desc_from_spec(jobs.spec_c1())
    mutate(jd)
    with pytest.raises(gxcorr.GxError) as ei:
        gxcorr.Correlator.from_desc(jd, device=-1)
    assert ei.value.status == status


def test_post_f_rotation_refused_for_complex_data():
    """Post-F (0th order) fringe rotation is real-data only (mode.cpp:1131-1134)."""
    jd = capi.job_desc_from_spec(jobs.spec_cplx8(fringe_rot_order=0))
    with pytest.raises(gxcorr.GxError) as ei:
        gxcorr.Correlator.from_desc(jd, device=-1)
    assert ei.value.status == 2
    c = gxcorr.Correlator.from_desc(capi.job_desc_from_spec(jobs.spec_c1(fringe_rot_order=0)), device=-1)
    c.close()


def test_tensor_core_xstep_limits():
    """The tensor-core X-step takes at most 128 station bands per freq
    (GX_ERR_UNSUPPORTED beyond), an unknown xstep is GX_ERR_ARG, and
    gx_set_tc_scales needs a device handle with that X-step (GX_ERR_STATE)."""
    from difx_b200.jobfiles import Subband
    big = jobs.JobSpec(name="tcbig", nstations=65, subbands=[Subband(6000.0, 16.0, "U", 64)], nbits=8,
                       sampling="COMPLEX", subint_ns=1_024_000, execute_seconds=2, max_delay_us=150.0, seed=1)
    with pytest.raises(gxcorr.GxError) as ei:
        gxcorr.Correlator.from_desc(capi.job_desc_from_spec(big, xstep=capi.GX_XSTEP_TC_FP16), device=-1)
    assert ei.value.status == 2
    ok = capi.job_desc_from_spec(jobs.spec_c1(), xstep=capi.GX_XSTEP_TC_FP16_HILO)
    c = gxcorr.Correlator.from_desc(ok, device=-1)
    with pytest.raises(gxcorr.GxError) as ei:
        c.set_tc_scales(0, 0, [1.0] * jobs.spec_c1().nchan)
    assert ei.value.status == 8
    c.close()
    bad = capi.job_desc_from_spec(jobs.spec_c1(), xstep=7)
    with pytest.raises(gxcorr.GxError) as ei:
        gxcorr.Correlator.from_desc(bad, device=-1)
    assert ei.value.status == 1


def test_missing_input_file_is_an_io_error():
    with pytest.raises(gxcorr.GxError) as ei:
        gxcorr.Correlator.from_input("/nonexistent/job.input", device=-1)
    assert ei.value.status == 5


def test_spectra_budget_sets_pass_length():
    """With a spectra budget the pass (block chunk) is the efficient length
    within the budget; an explicit block_chunk wins; the default fills 2 GB."""
    spec = jobs.spec_c2small()
    per_block = len(spec.subbands) * spec.nchan * 8
    lens = {}
    for budget in (0, 1 << 20, 64 << 20, 1 << 34):
        c = gxcorr.Correlator.from_desc(capi.job_desc_from_spec(spec, spectra_budget_bytes=budget), device=-1)
        lens[budget] = c.info.block_chunk
        c.close()
    assert lens[0] == spec.blocks_per_send                      # 2 GB holds the whole subint
    assert 16 <= lens[1 << 20] <= max(16, (1 << 20) // (per_block * spec.nstations * len(spec.pols)))
    assert lens[1 << 20] <= lens[64 << 20] <= lens[1 << 34] <= spec.blocks_per_send
    c = gxcorr.Correlator.from_desc(capi.job_desc_from_spec(spec, block_chunk=50, spectra_budget_bytes=1 << 20),
                                    device=-1)
    assert c.info.block_chunk == 50
    c.close()


def test_async_needs_a_device_handle():
    c = gxcorr.Correlator.from_desc(capi.job_desc_from_spec(jobs.spec_c1()), device=-1)
    out = np.zeros(c.result_length, np.complex64)
    with pytest.raises(gxcorr.GxError) as ei:
        c.subint_async(capi.SubintDesc(0, 0, 0, 0.0, [0] * 4, [0] * 4, [0] * 4, 3), out)
    assert ei.value.status == 8
    with pytest.raises(gxcorr.GxError) as ei:
        c.wait()
    assert ei.value.status == 8
    c.close()


def test_interlaced_vdif_input_matches_descriptor(tmp_path):
    """DATA FORMAT INTERLACEDVDIF/<threads> (configuration.cpp:1491-1498,
    2632-2651): the Core sees multiplexed frames of (per-thread frame - 32) x
    threads + 32 bytes; the .input and the descriptor give the same layout."""
    from difx_b200.jobfiles import write_job
    spec = jobs.spec_c1(name="mux_in", mux_threads=8)
    paths = write_job(spec, str(tmp_path))
    text = open(paths["input"]).read()
    assert "INTERLACEDVDIF/0:1:2:3:4:5:6:7" in text
    sizes = re.findall(r"^DATA FRAME SIZE:\s*(\d+)", text, re.M)
    assert sizes and all(int(x) == spec.payload_bytes // 8 + 32 for x in sizes)
    a = gxcorr.Correlator.from_input(paths["input"], device=-1)
    b = gxcorr.Correlator.from_desc(capi.job_desc_from_spec(spec), device=-1)
    assert a.info.result_length == b.info.result_length
    for x, y in zip(a.offsets(), b.offsets()):
        assert np.array_equal(x, y)
    assert a.info.blocks_per_send == b.info.blocks_per_send
    a.close()
    b.close()


def test_interlaced_vdif_band_limit():
    """Per-band EDV4 masks use int-width thread bits in the reference: more
    than 30 interlaced bands are refused."""
    from difx_b200.jobfiles import Subband
    spec = jobs.spec_c1(name="mux32", mux_threads=32, payload_bytes=8192,
                        subbands=[Subband(8400.0 + 16 * i, 16.0, "U", 128) for i in range(16)])
    with pytest.raises(gxcorr.GxError) as ei:
        gxcorr.Correlator.from_desc(capi.job_desc_from_spec(spec), device=-1)
    assert ei.value.status == 2


def test_sub_byte_time_samples():
    """Real time samples narrower than a byte open (sample granularity 8 /
    bits); complex ones are refused (the reference's granularity erase treats
    its complex unpack arrays as floats, mk5mode.cpp:118-141)."""
    from difx_b200.jobfiles import Subband
    ok = jobs.spec_c1(name="g2", subbands=[Subband(8400.0, 16.0, "U", 128)])
    assert ok.bits_per_timesample == 4
    gxcorr.Correlator.from_desc(capi.job_desc_from_spec(ok), device=-1).close()
    bad = jobs.spec_cplx8(name="gc", nbits=2, pols=("R",), subbands=[Subband(6000.0, 16.0, "U", 256)])
    with pytest.raises(gxcorr.GxError) as ei:
        gxcorr.Correlator.from_desc(capi.job_desc_from_spec(bad), device=-1)
    assert ei.value.status == 2
