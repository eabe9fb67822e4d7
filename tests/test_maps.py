"""SpatiallyExplicit map input: the native (Geo)TIFF loader and the
reference's map fix-ups (rustcoalescence/scenarios/src/spatially_explicit/
maps/), on CPU.

The loader is checked against the reference's own map fixtures
(maps/test, maps/madingley: LZW strips written by GDAL) decoded by PIL and
by an independent pure-Python reader, against synthetic maps in every
supported encoding, and on the reference's error cases; the fix-ups against
a numpy restatement of maps/mod.rs:90-215.
"""
import os

import numpy as np
import pytest
import tiff_util

REF_MAPS = os.environ.get("NECSIM_REFERENCE_MAPS", "")
needs_fixtures = pytest.mark.skipif(not REF_MAPS or not os.path.isdir(REF_MAPS),
                                    reason="set NECSIM_REFERENCE_MAPS to the reference's maps/ folder")


@needs_fixtures
def test_reference_habitat_fixture_matches_pil(nb):
    from PIL import Image
    for rel in ("test/habitat.tif", "madingley/fg0size8/habitat.tif", "madingley/fg0size9/habitat.tif",
                "madingley/fg0size12/habitat.tif"):
        got = nb.load_map(os.path.join(REF_MAPS, rel), "u32")
        want = np.array(Image.open(os.path.join(REF_MAPS, rel))).astype(np.int64)
        assert got.dtype == np.uint32 and got.shape == want.shape
        assert np.array_equal(got.astype(np.int64), want), rel


@needs_fixtures
def test_reference_f64_fixtures_match_python_reader(nb):
    for rel in ("test/dispersal.tif", "madingley/fg0size8/turnover.tif", "madingley/fg0size12/turnover.tif"):
        path = os.path.join(REF_MAPS, rel)
        got = nb.load_map(path, "f64", strict=True)
        want = tiff_util.read_tiff_strips(path)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), rel
    d = nb.load_map(os.path.join(REF_MAPS, "test/dispersal.tif"), "f64")
    assert d.shape == (1435, 1435)  # the 35 x 41 habitat map's cells squared
    assert np.allclose(d.sum(axis=1), 1.0)


@needs_fixtures
def test_reference_fixture_scenario_loads(nb):
    """maps/test as `SpatiallyExplicit(habitat, dispersal, mode: OffByOne)`."""
    sc = nb.spatially_explicit_from_maps(os.path.join(REF_MAPS, "test/habitat.tif"),
                                         os.path.join(REF_MAPS, "test/dispersal.tif"))
    assert sc.habitat.shape == (41, 35) and sc.dispersal.shape == (1435, 1435)
    assert int(sc.habitat.sum()) == 287933


@needs_fixtures
def test_habitat_loaded_as_f64_is_rejected(nb):
    with pytest.raises(nb.NecsimError, match="bitwidth"):
        nb.load_map(os.path.join(REF_MAPS, "test/habitat.tif"), "f64")
    with pytest.raises(nb.NecsimError, match="bitwidth"):
        nb.load_map(os.path.join(REF_MAPS, "test/dispersal.tif"), "u32")


ENCODINGS = [
    dict(),
    dict(compression=5),
    dict(compression=8),
    dict(compression=32946),
    dict(compression=32773),
    dict(compression=5, predictor=2),
    dict(compression=8, predictor=2, big=True),
    dict(big=True),
    dict(bigtiff=True, compression=5),
    dict(bigtiff=True, big=True, compression=32773),
    dict(rows_per_strip=3, compression=5),
    dict(rows_per_strip=1),
    dict(tile=(16, 16), compression=5),
    dict(tile=(32, 16), compression=8, predictor=2, big=True),
]


@pytest.mark.parametrize("enc", ENCODINGS, ids=lambda e: "-".join("%s%s" % kv for kv in e.items()) or "plain")
def test_synthetic_maps_round_trip(nb, tmp_path, enc):
    rng = np.random.default_rng(7)
    hab = rng.integers(0, 40, size=(37, 53), dtype=np.uint32)
    hab[rng.random(hab.shape) < 0.3] = 0
    hab[0, :5] = [0, 0xFFFFFFFF, 1, 2, 0x80000000]
    disp = rng.random((21, 45))
    disp[3, 4:9] = [0.0, -0.0, np.inf, 1e-310, 1e300]
    for arr, dtype in ((hab, "u32"), (disp, "f64")):
        p = tmp_path / ("m_%s.tif" % dtype)
        tiff_util.write_tiff(str(p), arr, **enc)
        got = nb.load_map(str(p), dtype, strict=True)
        assert got.shape == arr.shape
        assert np.array_equal(got.view(np.uint64 if dtype == "f64" else np.uint32),
                              arr.view(np.uint64 if dtype == "f64" else np.uint32))


@pytest.mark.parametrize("enc", [dict(predictor=3), dict(predictor=3, compression=5, big=True),
                                 dict(predictor=3, tile=(16, 16), compression=8)])
def test_floating_point_predictor(nb, tmp_path, enc):
    disp = np.random.default_rng(3).normal(size=(19, 33)) * 1e3
    p = tmp_path / "fp.tif"
    tiff_util.write_tiff(str(p), disp, **enc)
    assert np.array_equal(nb.load_map(str(p), "f64").view(np.uint64), disp.view(np.uint64))


def test_gdal_nodata(nb, tmp_path):
    hab = np.array([[7, 1, 7], [0, 9, 7]], dtype=np.uint32)
    p = tmp_path / "nd.tif"
    tiff_util.write_tiff(str(p), hab, nodata="7", compression=5)
    assert nb.load_map(str(p), "u32").tolist() == [[0, 1, 0], [0, 9, 0]]
    assert nb.load_map(str(p), "u32", strict=True).tolist() == hab.tolist()
    tiff_util.write_tiff(str(p), hab, nodata="+9")  # Rust's u32 parser takes a leading '+'
    assert nb.load_map(str(p), "u32").tolist() == [[7, 1, 7], [0, 0, 7]]
    for bad in ("abc", " 7", "7.0", "-1", "4294967296", ""):
        tiff_util.write_tiff(str(p), hab, nodata=bad)
        with pytest.raises(nb.NecsimError, match="nodata"):
            nb.load_map(str(p), "u32")
        assert nb.load_map(str(p), "u32", strict=True).tolist() == hab.tolist()
    d = np.array([[-3.4028234663852886e38, 0.5], [2.0, -3.4028234663852886e38]])
    tiff_util.write_tiff(str(p), d, nodata="-3.4028234663852886e+38")
    assert nb.load_map(str(p), "f64").tolist() == [[0.0, 0.5], [2.0, 0.0]]
    for text, value in (("inf", np.inf), ("-Infinity", -np.inf), ("1e0", 1.0), (".5", 0.5), ("2.", 2.0)):
        d2 = np.array([[value, 3.0]])
        tiff_util.write_tiff(str(p), d2, nodata=text)
        assert nb.load_map(str(p), "f64").tolist() == [[0.0, 3.0]], text
    tiff_util.write_tiff(str(p), np.array([[np.nan, 3.0]]), nodata="NaN")  # NaN equals nothing
    assert np.isnan(nb.load_map(str(p), "f64")[0, 0])
    for bad in ("0x1p3", "1e", "e5", " 1", "1 "):
        tiff_util.write_tiff(str(p), d, nodata=bad)
        with pytest.raises(nb.NecsimError, match="nodata"):
            nb.load_map(str(p), "f64")


@pytest.mark.parametrize("kw,msg", [
    (dict(spp=3), "one sample per pixel"),
    (dict(photometric=None), "PhotometricInterpretation"),
    (dict(photometric=2), "not Gray"),
    (dict(compression=7), "compression"),
])
def test_unsupported_layouts_are_rejected(nb, tmp_path, kw, msg):
    hab = np.arange(12, dtype=np.uint32).reshape(3, 4)
    p = tmp_path / "bad.tif"
    if kw.get("compression") == 7:
        tiff_util.write_tiff(str(p), hab)
        raw = bytearray(p.read_bytes())
        # patch the Compression tag's value in place (entry 259, SHORT 1 -> 7)
        at = raw.find(b"\x03\x01\x03\x00\x01\x00\x00\x00\x01\x00")
        raw[at + 8] = 7
        p.write_bytes(bytes(raw))
    elif kw.get("spp") == 3:
        tiff_util.write_tiff(str(p), hab, spp=3)
    else:
        tiff_util.write_tiff(str(p), hab, **kw)
    with pytest.raises(nb.NecsimError, match=msg):
        nb.load_map(str(p), "u32")


def test_sample_format_checks(nb, tmp_path):
    p = tmp_path / "sf.tif"
    tiff_util.write_tiff(str(p), np.arange(6, dtype=np.int32).reshape(2, 3))  # SampleFormat Int
    with pytest.raises(nb.NecsimError, match="sample format"):
        nb.load_map(str(p), "u32")
    tiff_util.write_tiff(str(p), np.arange(6, dtype=np.uint32).reshape(2, 3), sample_format=False)
    assert nb.load_map(str(p), "u32").tolist() == [[0, 1, 2], [3, 4, 5]]  # absent: Uint
    tiff_util.write_tiff(str(p), np.arange(6, dtype=np.uint64).reshape(2, 3))  # 64-bit Uint
    with pytest.raises(nb.NecsimError, match="sample format"):
        nb.load_map(str(p), "f64")
    tiff_util.write_tiff(str(p), np.ones((2, 3)), sample_format=False)  # 64-bit, no format: not f64
    with pytest.raises(nb.NecsimError, match="f64"):
        nb.load_map(str(p), "f64")


def test_broken_files_are_rejected(nb, tmp_path):
    p = tmp_path / "x.tif"
    p.write_bytes(b"not a tiff at all")
    with pytest.raises(nb.NecsimError, match="not a TIFF"):
        nb.load_map(str(p), "u32")
    tiff_util.write_tiff(str(p), np.arange(400, dtype=np.uint32).reshape(20, 20), compression=5)
    raw = p.read_bytes()
    p.write_bytes(raw[:40])  # the IFD is gone
    with pytest.raises(nb.NecsimError, match="truncated"):
        nb.load_map(str(p), "u32")
    with pytest.raises(nb.NecsimError, match="could not read"):
        nb.load_map(str(tmp_path / "missing.tif"), "u32")


# ---- fix-ups (maps/mod.rs) restated with numpy ----
def fix_restated(hab, disp, turnover, mode):
    hab, disp = hab.copy(), disp.copy()
    if mode == "Strict":
        return hab, disp
    w = hab.shape[1]
    for cell in range(hab.size):
        y, x = divmod(cell, w)
        if hab[y, x] <= 1:  # fix_habitat_map
            if turnover is not None and turnover[y, x] == 0.0:
                hab[y, x] = 0
            elif cell < disp.shape[0] and (disp[cell] > 0.0).any():
                hab[y, x] = 1
            else:
                hab[y, x] = 0
    if mode == "OffByOne":
        return hab, disp
    if turnover is not None:  # fix_no_turnover_habitat_map
        hab[turnover == 0.0] = 0
    flat = hab.reshape(-1)
    for row in range(flat.size):  # fix_dispersal_map
        if flat[row] == 0:
            disp[row][disp[row] > 0.0] = 0.0
        else:
            disp[row][(flat == 0) & (disp[row] > 0.0)] = 0.0
            total = 0.0
            for v in disp[row]:
                total += v
            if total <= 0.0:
                disp[row, row] = 1.0
    return hab, disp


@pytest.mark.parametrize("mode", ["OffByOne", "FixMe", "Strict"])
@pytest.mark.parametrize("with_turnover", [False, True])
def test_fixups_match_restatement(nb, mode, with_turnover):
    rng = np.random.default_rng(11)
    h, w = 9, 7
    hab = rng.integers(0, 4, size=(h, w)).astype(np.uint32)
    disp = rng.random((h * w, h * w)) * (rng.random((h * w, h * w)) < 0.2)
    disp[5] = 0.0           # a cell with no dispersal at all
    disp[hab.reshape(-1) == 0, 0] = 0.3  # dispersal from non-habitat
    turnover = None
    if with_turnover:
        turnover = rng.random((h, w)) * (rng.random((h, w)) < 0.8)
    got = nb.fix_maps(hab, disp, turnover, mode)
    want = fix_restated(hab, disp, turnover, mode)
    assert np.array_equal(got[0], want[0])
    assert np.array_equal(got[1].view(np.uint64), want[1].view(np.uint64))
    if mode != "Strict":
        assert not np.array_equal(got[0], hab)


def test_fixups_reject_negative_maps_and_bad_shapes(nb):
    hab = np.ones((2, 2), dtype=np.uint32)
    disp = np.eye(4)
    disp[1, 2] = -1e-300
    with pytest.raises(nb.NecsimError, match="non-negative"):
        nb.fix_maps(hab, disp, None, "Strict")
    with pytest.raises(nb.NecsimError, match="Turnover"):
        nb.fix_maps(hab, np.eye(4), -np.ones((2, 2)), "OffByOne")
    with pytest.raises(nb.NecsimError, match="width"):
        nb.fix_maps(hab, np.eye(3), None, "FixMe")
    nb.fix_maps(hab, np.eye(3), None, "OffByOne")  # only FixMe indexes the map as (w*h)^2
    with pytest.raises(ValueError):
        nb.fix_maps(hab, np.eye(4), None, "Lenient")


def test_corrupt_counts_and_sizes_are_rejected(nb, tmp_path):
    import struct
    p = tmp_path / "c.tif"
    tiff_util.write_tiff(str(p), np.arange(12, dtype=np.uint32).reshape(3, 4))
    raw = bytearray(p.read_bytes())
    (ifd,) = struct.unpack("<I", raw[4:8])
    (n,) = struct.unpack("<H", raw[ifd:ifd + 2])
    entries = {struct.unpack("<H", raw[ifd + 2 + 12 * j: ifd + 4 + 12 * j])[0]: ifd + 2 + 12 * j for j in range(n)}
    bad = bytearray(raw)
    bad[entries[273] + 4: entries[273] + 8] = struct.pack("<I", 0x7FFFFFFF)  # StripOffsets count
    p.write_bytes(bytes(bad))
    with pytest.raises(nb.NecsimError, match="truncated"):
        nb.load_map(str(p), "u32")
    bad = bytearray(raw)
    bad[entries[256] + 8: entries[256] + 12] = struct.pack("<I", 0xFFFFFFFF)  # ImageWidth
    bad[entries[257] + 8: entries[257] + 12] = struct.pack("<I", 0xFFFFFFFF)  # ImageLength
    p.write_bytes(bytes(bad))
    with pytest.raises(nb.NecsimError, match="too large"):
        nb.load_map(str(p), "u32")
