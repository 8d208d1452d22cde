"""The source-CAMBI cache (es_cambi_cache_*, the reference's CambiCache, src/cache.cpp:13-88) and the per-frame JSON
(src/main.cpp:767-774) on the CPU: the file name against an independent restatement of the key (FNV-1a of the key text
and the first and last MiB), records across the 240-record flushes, a torn tail record dropped on reopening, keys that
follow the content and not the path, frames without timestamps never cached, and the JSON digits."""

import os
import shutil
import struct

import numpy as np

import es_b200

NO_PTS = -(1 << 63)


def fnv1a(h, data):
    for b in data:
        h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def expected_name(path, x0, y0, w, h, depth):
    data = open(path, "rb").read()
    size = len(data)
    key = f"cambi 1 {size} {x0} {y0} {w} {h} {depth}".encode()
    hsh = fnv1a(0xCBF29CE484222325, key)
    mib = 1 << 20
    hsh = fnv1a(hsh, data[:mib])
    start = max(size - mib, 0)
    hsh = fnv1a(hsh, data[start:start + mib])
    return f"{hsh:016x}.cambi"


def make_source(tmp_path, name, size, seed):
    p = tmp_path / name
    p.write_bytes(np.random.default_rng(seed).integers(0, 256, size, dtype=np.uint8).tobytes())
    return str(p)


def test_key_and_records_round_trip(tmp_path):
    src = make_source(tmp_path, "source.mkv", 2_500_000, 1)
    d = str(tmp_path / "cache")
    c = es_b200.CambiCache(src, 0, 140, 1920, 800, 10, d)
    assert os.path.basename(c.file) == expected_name(src, 0, 140, 1920, 800, 10)
    for i in range(500):
        c.add(1000 * i, 0.25 * i)
    c.add(NO_PTS, 9.0)
    assert c.find(1000 * 7) == 1.75 and c.find(NO_PTS) is None and c.find(3) is None
    c.close()
    assert os.path.getsize(os.path.join(d, expected_name(src, 0, 140, 1920, 800, 10))) == 500 * 16
    c = es_b200.CambiCache(src, 0, 140, 1920, 800, 10, d)
    assert all(c.find(1000 * i) == 0.25 * i for i in range(500))
    c.close()


def test_torn_tail_record_is_dropped(tmp_path):
    src = make_source(tmp_path, "a.mp4", 100_000, 2)
    d = str(tmp_path / "cache")
    c = es_b200.CambiCache(src, 0, 0, 640, 360, 8, d)
    for i in range(10):
        c.add(i, float(i))
    path = c.file
    c.close()
    with open(path, "ab") as f:
        f.write(struct.pack("<q", 77)[:7])  # a run stopped in the middle of a record
    c = es_b200.CambiCache(src, 0, 0, 640, 360, 8, d)
    assert os.path.getsize(path) == 160 and c.find(9) == 9.0 and c.find(77) is None
    c.add(10, 10.0)
    c.close()
    c = es_b200.CambiCache(src, 0, 0, 640, 360, 8, d)
    assert c.find(10) == 10.0
    c.close()


def test_key_follows_content_crop_and_depth(tmp_path):
    src = make_source(tmp_path, "x.mkv", 3_000_000, 3)
    moved = str(tmp_path / "renamed.mkv")
    shutil.copy(src, moved)
    d = str(tmp_path / "cache")
    names = set()
    for args in ((src, 0, 0, 1920, 1080, 10), (moved, 0, 0, 1920, 1080, 10), (src, 0, 0, 1920, 1080, 8), (src, 0, 140, 1920, 800, 10)):
        c = es_b200.CambiCache(*args, d)
        names.add(os.path.basename(c.file))
        c.close()
    assert len(names) == 3  # the renamed copy shares the first key


def test_unopenable_cache_keeps_nothing(tmp_path):
    c = es_b200.CambiCache(str(tmp_path / "missing.mkv"), 0, 0, 64, 64, 10, str(tmp_path / "cache"))
    assert c.file == ""
    c.add(1, 2.0)
    assert c.find(1) is None
    c.close()


def test_per_frame_json_digits():
    cambi = [0.0, 1.23456789, 12.5]
    src = [0.5, 0.25, 3.0]
    psnr = [40.12345, 38.0, 99.9996]
    got = es_b200.per_frame_json(cambi, src, psnr)
    want = ('{"vmaf": null, "cambi": [0.000000,1.234568,12.500000], "cambi_source": [0.500000,0.250000,3.000000], '
            '"psnr_y": [40.123,38.000,100.000]}')
    assert got == want
    assert es_b200.per_frame_json(cambi, src, psnr, vmaf=[95.1, 96.2, 97.3]).startswith('{"vmaf": [95.100000,96.200000,97.300000]')
