"""C ABI surface on a CPU-only host: the library loads, exports every symbol
the public headers declare, and its host-side calls honour the reference's
formats and error behaviour (no GPU compute here)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import graphindor_b200 as gi
from graphindor_b200 import _native as N

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(gi_[a-z_0-9]+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported(native):
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(native, n)]
    assert not missing, missing


def test_status_strings(native):
    assert native.gi_status_string(0) == b"ok"
    assert b"connected" in native.gi_status_string(N.GI_EDISCONNECTED)
    assert native.gi_version() >= 1


def test_g_roundtrip_and_checksum(tmp_path, native):
    g = gi.gen.rmat(7, 4.0, 3) if hasattr(gi, "gen") else None
    from graphindor_b200 import gen
    g = gen.rmat(7, 4.0, 3)
    p = tmp_path / "x.g"
    gi.write_g(str(p), g.vertex, g.edge, g.max_intersection_size, 1234)
    raw = p.read_bytes()
    assert len(raw) == 32 + 8 * (g.v_cnt + 1) + 4 * g.e_cnt
    words = np.frombuffer(raw[:32], dtype=np.uint32)
    assert int(words.sum(dtype=np.uint64)) % (1 << 32) == 0  # header words sum to zero
    v, e, mi, tri = gi.read_g(str(p))
    assert np.array_equal(v, g.vertex) and np.array_equal(e, g.edge)
    assert mi == g.max_intersection_size and tri == 1234
    bad = bytearray(raw)
    bad[8] ^= 1
    (tmp_path / "bad.g").write_bytes(bytes(bad))
    with pytest.raises(gi.GIError) as ei:
        gi.read_g(str(tmp_path / "bad.g"))
    assert ei.value.status == N.GI_EIO
    (tmp_path / "short.g").write_bytes(raw[:-4])
    with pytest.raises(gi.GIError) as ei:
        gi.read_g(str(tmp_path / "short.g"))
    assert ei.value.status == N.GI_EIO
    with pytest.raises(gi.GIError) as ei:
        gi.read_g(str(tmp_path / "missing.g"))
    assert ei.value.status == N.GI_EIO


@pytest.mark.parametrize("n,adj,status", [
    (8, "0" * 64, N.GI_EINVAL),
    (2, "0110", N.GI_EINVAL),
    (4, "011", N.GI_EINVAL),
    (4, "0100100000010010", N.GI_EDISCONNECTED),
])
def test_plan_errors(native, n, adj, status):
    h = C.c_void_p()
    rc = native.gi_plan_create(n, adj.encode(), 1000, 5000, 0, 1, 1, C.byref(h))
    assert rc == status
    assert not h


def test_motif_numbers(native):
    assert [native.gi_motif_num(k) for k in range(3, 8)] == [2, 6, 21, 112, 853]
    assert native.gi_motif_num(8) == -1


def test_explicit_plan_counts_are_self_consistent(native):
    # An explicit schedule gets fresh IEP tables and its own redundancy.
    p = gi.Pattern(4, "0111101111001100")
    s = gi.Schedule_IEP(p, order=[0, 1, 2, 3], restricts=[(2, 3)], enable_iep=True)
    d = s.export()
    assert d["in_exclusion_optimize_num"] == 2
    assert d["redundancy"] >= 1
