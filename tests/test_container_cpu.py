"""The container fixtures (written by the reference's CPU path) against the
oracle's OpenMP layout at one thread, and their footers and tables."""
import json
import os
import struct

import numpy as np
import pytest

import synth

HERE = os.path.join(os.path.dirname(__file__), "golden", "containers")
MANIFEST = json.load(open(os.path.join(HERE, "manifest.json")))


def _field(m):
    d = synth.small_field(tuple(m["dims"]), seed=m["seed"], kind=m["kind"])
    return (d * np.float32(m["scale"])).astype(np.float32)


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_container_fixture(ora, name):
    m = MANIFEST[name]
    blob = open(os.path.join(HERE, name), "rb").read()
    ts, ss = struct.unpack("<QQ", blob[-16:])
    assert ts == m["topo_bytes"] and ss == m["sort_bytes"] and ts + ss + 16 == len(blob)
    T = m["threads"]
    table = struct.unpack("<%dQ" % T, blob[: 8 * T])
    assert table[0] == 0 and list(table) == sorted(table)
    if T == 1:
        d = _field(m)
        eb, B = m["eb"], m["block_size"]
        cp = ora.sort_cp(ora.find_cp(d, eb), d)
        assert blob[:ts] == ora.encode_topo(d, eb, B, ora.mark_types(cp, d.shape), cpu_layout=True)
        sp = ora.extract_sp(cp)
        assert blob[ts:ts + ss] == (ora.encode_ints(sp, B, cpu_layout=True) if len(sp) else b"")
