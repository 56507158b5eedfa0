"""Host side of the tile autotuner's interface, without a GPU: the Python
mirror reads ns3d_autotune's timing array (NS3D_TUNE_TIMES doubles, tile t
of family f at 5 f + t, -1 for a tile not timed) into per-family dicts, and
the header's constants match the mirror's."""
import ctypes
import os
import re

from ns3dperiodic_b200 import solver as S

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "ns3d.h")


def _define(name):
    m = re.search(rf"#define\s+{name}\s+(\d+)", open(HEADER).read())
    assert m, name
    return int(m.group(1))


def test_header_constants_match_the_mirror():
    assert _define("NS3D_TILES_PER_FAMILY") == S.TILES_PER_FAMILY
    assert _define("NS3D_TILE_FAMILIES") == 4
    assert _define("NS3D_TUNE_TIMES") == 4 * S.TILES_PER_FAMILY


def test_autotune_reads_the_timing_array():
    # family 0: tiles 0, 1, 4; family 1: 0, 1, 2, 4; family 2: 0, 3; family 3: 0, 1
    filled = {0: 0.30, 1: 0.26, 4: 0.25, 5: 0.55, 6: 0.50, 7: 0.54, 9: 0.49,
              10: 0.18, 13: 0.17, 15: 0.30, 16: 0.44}
    chosen = [4, 4, 3, 0]

    def fake_autotune(h, reps, force, ms):
        for i in range(4 * S.TILES_PER_FAMILY):
            ms[i] = filled.get(i, -1.0)
        return 0

    def fake_get(h, t):
        for f in range(4):
            t[f] = chosen[f]
        return 0

    def check(rc, where):
        assert rc == 0, where

    r = S._autotune(fake_autotune, None, check, 5, False, fake_get)
    assert r["tiles"] == chosen
    assert r["ms"] == [{0: 0.30, 1: 0.26, 4: 0.25}, {0: 0.55, 1: 0.50, 2: 0.54, 4: 0.49},
                       {0: 0.18, 3: 0.17}, {0: 0.30, 1: 0.44}]


def test_autotune_without_timing_reports_none():
    def cached(h, reps, force, ms):
        for i in range(4 * S.TILES_PER_FAMILY):
            ms[i] = -1.0
        return 0

    def get(h, t):
        for f in range(4):
            t[f] = 0
        return 0

    r = S._autotune(cached, None, lambda rc, w: None, 5, False, get)
    assert r == {"tiles": [0, 0, 0, 0], "ms": None}
