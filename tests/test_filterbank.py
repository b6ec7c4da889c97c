"""SIGPROC filterbank ingest (read_filterbank, src/gaffa/io/filterbank.cpp).

Known-answer cases restate tests/cpp/test_filterbank.cpp of the reference with
fixtures written here; tests/golden/ref_filterbank.npz holds the reference's
own reading of its tests/data/basetest.fil (tests/golden/make_golden.py).
"""
import hashlib
import struct
from pathlib import Path

import numpy as np
import pytest

from gaffa_b200 import core

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_filterbank.npz"


def _reference_fil() -> Path:
    """basetest.fil under the reference checkout the checkers are built from
    (GAFFA_REFERENCE_DIR, as __graft_entry__.build uses it)."""
    import __graft_entry__
    return Path(__graft_entry__.REFERENCE_DIR) / "tests" / "data" / "basetest.fil"


REFERENCE_FIL = _reference_fil()


def _s(b: bytearray, text: str):
    raw = text.encode()
    b += struct.pack("<i", len(raw)) + raw


def write_fil(path, samples: np.ndarray, nbits=8, nifs=1, nchans=4, fch1=1000.0, foff=1.0, tsamp=1.0,
              frequency_table=None, rawdatafile=None, optional=None):
    """Test fixture writer following test_filterbank.cpp:42-107."""
    b = bytearray()
    _s(b, "HEADER_START")
    if rawdatafile:
        _s(b, "rawdatafile")
        _s(b, rawdatafile)
    _s(b, "source_name")
    _s(b, "test-source")
    for k, v in (("telescope_id", 0), ("machine_id", 0), ("data_type", 1), ("nifs", nifs), ("nchans", nchans),
                 ("nbits", nbits)):
        _s(b, k)
        b += struct.pack("<i", v)
    for k, v in (("tsamp", tsamp), ("tstart", 0.0)):
        _s(b, k)
        b += struct.pack("<d", v)
    for k, v in (optional or {}).items():
        _s(b, k)
        b += struct.pack("<d" if isinstance(v, float) else "<i", v)
    if frequency_table is None:
        for k, v in (("fch1", fch1), ("foff", foff)):
            _s(b, k)
            b += struct.pack("<d", v)
    else:
        _s(b, "FREQUENCY_START")
        for f in frequency_table:
            _s(b, "fchannel")
            b += struct.pack("<d", f)
        _s(b, "FREQUENCY_END")
    _s(b, "HEADER_END")
    Path(path).write_bytes(bytes(b) + np.ascontiguousarray(samples).tobytes())
    return path


def test_positive_foff_reads_directly(tmp_path):
    p = write_fil(tmp_path / "a.fil", np.arange(1, 9, dtype=np.uint8))
    h, f, x = core.read_filterbank(p)
    assert (h["nsamples"], h["nchans"], h["fch1"], h["foff"], h["reversed"]) == (2, 4, 1000.0, 1.0, 0)
    assert list(x.ravel()) == [1, 2, 3, 4, 5, 6, 7, 8]
    assert list(f) == [1000.0, 1001.0, 1002.0, 1003.0]


def test_negative_foff_normalised_to_ascending(tmp_path):
    p = write_fil(tmp_path / "a.fil", np.arange(1, 9, dtype=np.uint8), foff=-1.0)
    h, f, x = core.read_filterbank(p)
    assert (h["fch1"], h["foff"], h["reversed"]) == (997.0, 1.0, 1)
    assert list(f) == [997.0, 998.0, 999.0, 1000.0]
    assert list(x.ravel()) == [4, 3, 2, 1, 8, 7, 6, 5]


def test_preserve_file_order(tmp_path):
    p = write_fil(tmp_path / "a.fil", np.arange(1, 5, dtype=np.uint8), foff=-1.0)
    h, f, x = core.read_filterbank(p, preserve_file_order=True)
    assert (h["fch1"], h["foff"]) == (1000.0, -1.0)
    assert list(f) == [1000.0, 999.0, 998.0, 997.0]
    assert list(x.ravel()) == [1, 2, 3, 4]


def test_each_if_reversed_independently(tmp_path):
    p = write_fil(tmp_path / "a.fil", np.array([1, 2, 3, 10, 11, 12], np.uint16), nbits=16, nifs=2, nchans=3,
                  fch1=100.0, foff=-2.0)
    _, _, x = core.read_filterbank(p)
    assert x.dtype == np.uint16 and list(x.ravel()) == [3, 2, 1, 12, 11, 10]


def test_float_samples(tmp_path):
    p = write_fil(tmp_path / "a.fil", np.array([1.5, 2.5], np.float32), nbits=32, nchans=2, fch1=10.0, foff=-0.5)
    _, _, x = core.read_filterbank(p)
    assert list(x.ravel()) == [2.5, 1.5]


def test_frequency_tables(tmp_path):
    p = write_fil(tmp_path / "d.fil", np.array([7, 8, 9], np.uint8), nchans=3, frequency_table=[30.0, 20.0, 10.0])
    h, f, x = core.read_filterbank(p)
    assert h["uses_frequency_table"] and h["fch1"] == 10.0
    assert list(f) == [10.0, 20.0, 30.0] and list(x.ravel()) == [9, 8, 7]
    p = write_fil(tmp_path / "e.fil", np.array([7, 8, 9], np.uint8), nchans=3, frequency_table=[10.0, 20.0, 30.0])
    h, f, x = core.read_filterbank(p)
    assert (h["fch1"], h["foff"]) == (0.0, 0.0)
    assert list(f) == [10.0, 20.0, 30.0] and list(x.ravel()) == [7, 8, 9]


def test_optional_fields(tmp_path):
    opt = {"barycentric": 1, "pulsarcentric": 2, "ibeam": 3, "nbeams": 4, "nbins": 5, "npuls": 6,
           "az_start": 11.5, "za_start": 12.5, "src_raj": 13.5, "src_dej": 14.5, "period": 15.5, "refdm": 16.5,
           "nsamples": 123456}
    p = write_fil(tmp_path / "a.fil", np.arange(4, dtype=np.uint8), rawdatafile="raw.dat", optional=opt)
    h, _, _ = core.read_filterbank(p)
    assert h["rawdatafile"] == "raw.dat" and h["source_name"] == "test-source"
    for k, v in opt.items():
        if k != "nsamples":
            assert h[k] == v
    assert h["nsamples"] == 1


def test_partial_row_range(tmp_path):
    x = np.arange(40, dtype=np.uint8)
    p = write_fil(tmp_path / "a.fil", x, foff=-1.0)
    _, _, part = core.read_filterbank(p, row_begin=3, nrows=4)
    assert np.array_equal(part.reshape(4, 4), x.reshape(10, 4)[3:7, ::-1])


def test_packed_two_bit_rows_reverse_fieldwise(tmp_path):
    rng = np.random.default_rng(3)
    levels = rng.integers(0, 4, size=(5, 8), dtype=np.uint8)          # 5 rows x 8 channels
    packed = np.zeros((5, 2), np.uint8)
    for c in range(8):
        packed[:, c // 4] |= levels[:, c] << (2 * (c % 4))
    p = write_fil(tmp_path / "a.fil", packed, nbits=2, nchans=8, foff=-1.0)
    h, _, x = core.read_filterbank(p)
    assert h["nsamples"] == 5 and x.shape == (5, 1, 2)
    got = np.stack([(x[:, 0, c // 4] >> (2 * (c % 4))) & 3 for c in range(8)], axis=1)
    assert np.array_equal(got, levels[:, ::-1])


@pytest.mark.parametrize("blob,msg", [
    (struct.pack("<i", 4) + b"NOPE", "HEADER_START"),
    (struct.pack("<i", 12) + b"HEADER_START" + struct.pack("<i", 5) + b"bogus", "Unknown filterbank header field"),
])
def test_malformed_headers(tmp_path, blob, msg):
    p = tmp_path / "bad.fil"
    p.write_bytes(blob)
    with pytest.raises(RuntimeError, match=msg):
        core.read_filterbank_header(p)


def test_rejects_partial_rows_and_bad_nbits(tmp_path):
    p = write_fil(tmp_path / "a.fil", np.arange(6, dtype=np.uint8))
    with pytest.raises(RuntimeError, match="whole number of rows"):
        core.read_filterbank_header(p)
    p = write_fil(tmp_path / "b.fil", np.arange(8, dtype=np.uint8), nbits=12)
    with pytest.raises(RuntimeError, match="nbits"):
        core.read_filterbank_header(p)


def test_reference_basetest_golden():
    if not REFERENCE_FIL.exists():
        pytest.skip("reference test data not present")
    g = np.load(GOLDEN)
    for tag, preserve in (("asc", False), ("file", True)):
        h, f, x = core.read_filterbank(REFERENCE_FIL, preserve_file_order=preserve)
        for k in h:
            key = f"{tag}_h_{k}"
            if key in g:
                assert h[k] == g[key][()], k
        assert np.array_equal(f, g[f"{tag}_freq"])
        raw = x.tobytes()
        assert hashlib.sha256(raw).hexdigest() == str(g[f"{tag}_digest"])
        assert raw[: len(g[f"{tag}_head"])] == g[f"{tag}_head"].tobytes()


def test_matches_reference_reader(tmp_path):
    from oracle.oracle import Oracle
    if not Oracle.available("reference"):
        pytest.skip("reference checker not built")
    ref = Oracle("reference")
    rng = np.random.default_rng(11)
    cases = [dict(nbits=8, nifs=1, nchans=16, foff=-0.5), dict(nbits=16, nifs=2, nchans=5, foff=-1.0),
             dict(nbits=32, nifs=1, nchans=7, foff=2.0), dict(nbits=8, nchans=4, frequency_table=[4.0, 3.0, 2.0, 1.0])]
    for i, kw in enumerate(cases):
        dt = {8: np.uint8, 16: np.uint16, 32: np.float32}[kw.get("nbits", 8)]
        n = kw.get("nifs", 1) * kw.get("nchans", 4) * 9
        data = (rng.random(n) * 200).astype(dt)
        p = write_fil(tmp_path / f"c{i}.fil", data, **kw)
        for preserve in (False, True):
            h, f, x = core.read_filterbank(p, preserve_file_order=preserve)
            rh, rf, rx = ref.read_filterbank(p, preserve)
            assert np.array_equal(f, rf) and x.tobytes() == rx.tobytes()
            for k in rh:
                assert h[k] == rh[k], k


@pytest.mark.gpu
@pytest.mark.parametrize("nbits", [8, 16, 32, 2])
def test_device_load_matches_host_read(tmp_path, nbits):
    rng = np.random.default_rng(nbits)
    nchans, nifs, nrows = 64, (2 if nbits == 16 else 1), 1000
    if nbits == 2:
        data = rng.integers(0, 256, size=nrows * nchans // 4, dtype=np.uint8)
    else:
        dt = {8: np.uint8, 16: np.uint16, 32: np.float32}[nbits]
        data = (rng.random(nrows * nifs * nchans) * 250).astype(dt)
    p = write_fil(tmp_path / "a.fil", data, nbits=nbits, nifs=nifs, nchans=nchans, foff=-0.25)
    for preserve in (False, True):
        _, _, host = core.read_filterbank(p, preserve_file_order=preserve)
        # a bounce buffer of a few rows forces many overlapped chunks
        _, _, dev = core.load_filterbank(p, preserve_file_order=preserve, bounce_bytes=4096)
        assert dev.cpu().numpy().tobytes() == host.tobytes()
    _, _, part = core.load_filterbank(p, row_begin=17, nrows=300, bounce_bytes=1 << 20)
    _, _, hpart = core.read_filterbank(p, row_begin=17, nrows=300)
    assert part.cpu().numpy().tobytes() == hpart.tobytes()
