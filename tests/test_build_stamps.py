"""The native build rebuilds an object whenever the contents of its inputs or
its command line differ from what it was built from, whatever the files'
modification times (an object compiled while a header was being edited is
never taken as current)."""
import os

from parahpop_b200 import build as B


def test_stamp_tracks_contents_not_mtimes(tmp_path):
    src, hdr, out = tmp_path / "a.cu", tmp_path / "a.cuh", tmp_path / "a.o"
    src.write_text("int a;")
    hdr.write_text("struct S { int x; };")
    cmd = ["true", str(src)]
    assert B._stale(out, cmd, [src, hdr])  # never built
    out.write_text("object")
    (tmp_path / "a.o.sha").write_text(B._digest(cmd, [src, hdr]))
    assert not B._stale(out, cmd, [src, hdr])
    # header edited, object newer than the edit: still stale
    hdr.write_text("struct S { int x; double y; };")
    os.utime(out, (os.path.getmtime(hdr) + 100,) * 2)
    assert B._stale(out, cmd, [src, hdr])
    # a different command line (other macros) is stale as well
    hdr.write_text("struct S { int x; };")
    assert not B._stale(out, cmd, [src, hdr])
    assert B._stale(out, cmd + ["-DX=1"], [src, hdr])
