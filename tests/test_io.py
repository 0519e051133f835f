"""CPU tests of the field-file I/O (sx_field_write / sx_field_read): the
reference's format -- a 10-line ASCII header (src/data2df.cpp:503-535) and
the fields' planes in binary, field after field (src/auxfield.cpp:997-1095)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def sx():
    import semtex_b200
    return semtex_b200


def _fields(seed=1, nz=3, nel=5, np_=4):
    rng = np.random.default_rng(seed)
    return {c: rng.standard_normal((nz, nel * np_ * np_)) for c in "uvp"}


def test_round_trip_and_header_text(sx, tmp_path):
    f = _fields()
    path = tmp_path / "run.fld"
    sx.write_field(path, f, 4, 5, session="channel", step=120, time=0.25, dt=1e-3, kinvis=5e-4, beta=1.0)
    lines = path.read_bytes().split(b"\n")[:10]
    labels = [b"Session", b"Created", b"Nr, Ns, Nz, Elements", b"Step", b"Time", b"Time step", b"Kinvis",
              b"Beta", b"Fields written", b"Format"]
    for ln, lab in zip(lines, labels):
        assert ln.rstrip().endswith(lab), (ln, lab)
    assert lines[0].startswith(b"channel ")
    assert lines[2].split()[:4] == [b"4", b"4", b"3", b"5"]
    assert lines[8].startswith(b"uvp ")
    assert b"binary IEEE little-endian" in lines[9]
    # the data: 3 fields x 3 planes x 80 doubles right after the header
    header_len = sum(len(x) + 1 for x in lines)
    assert path.stat().st_size == header_len + 3 * 3 * 80 * 8
    h, g = sx.read_field(path)
    assert (h["np"], h["nz"], h["nel"], h["step"], h["fields"], h["swapped"]) == (4, 3, 5, 120, "uvp", 0)
    assert h["session"] == "channel" and abs(h["time"] - 0.25) < 1e-12 and abs(h["kinvis"] - 5e-4) < 1e-15
    for c in "uvp":
        assert np.array_equal(g[c], f[c])


def test_big_endian_file_is_swapped(sx, tmp_path):
    f = _fields(seed=2, nz=2, nel=3, np_=5)
    path = tmp_path / "be.fld"
    hdr = ["%-25s Session" % "be", "%-25s Created" % "Thu Jan 01 00:00:00 1970",
           "%-5d %-5d %-5d %-5d   Nr, Ns, Nz, Elements" % (5, 5, 2, 3), "%-25d Step" % 7,
           "%-25.6g Time" % 1.5, "%-25.6g Time step" % 0.01, "%-25.6g Kinvis" % 0.1, "%-25.6g Beta" % 2.0,
           "%-25s Fields written" % "uvp", "%-25s Format" % "binary IEEE big-endian"]
    data = b"".join(f[c].astype(">f8").tobytes() for c in "uvp")
    path.write_bytes(("\n".join(hdr) + "\n").encode() + data)
    h, g = sx.read_field(path)
    assert h["swapped"] == 1 and h["step"] == 7 and h["fields"] == "uvp"
    for c in "uvp":
        assert np.array_equal(g[c], f[c])


def test_not_a_field_file_is_refused(sx, tmp_path):
    path = tmp_path / "junk.fld"
    path.write_bytes(b"hello\n" * 12)
    with pytest.raises(sx.SolverError):
        sx.read_field(path)
    short = tmp_path / "short.fld"
    sx.write_field(short, _fields(), 4, 5)
    short.write_bytes(short.read_bytes()[:-8])
    with pytest.raises(sx.SolverError):
        sx.read_field(short)


def _channel_pair(renumber="rcm"):
    from semtex_b200.mesh import rect_mesh
    kw = dict(x0=0.0, x1=2 * np.pi, y0=0.0, y1=1.0, jitter=0.15, seed=2, periodic_x=True, renumber=renumber)
    mu = rect_mesh(6, 4, 5, bc={"bottom": "D", "top": "D"}, **kw)   # velocity: Dirichlet walls
    mp = rect_mesh(6, 4, 5, bc={"bottom": "N", "top": "N"}, **kw)   # pressure: natural walls
    return mu, mp


def test_numbering_round_trip_two_sets(sx, tmp_path):
    """Two number sets, as enumerate writes them for "uvp" (utility/
    enumerate.cpp:426-537): "uv" with essential walls, "p" without."""
    mu, mp = _channel_pair()
    path = tmp_path / "chan.num"
    sx.write_numbering(path, {"uv": mu, "p": mp}, fields="uvp")
    text = path.read_text().splitlines()
    assert text[0].split() == ["#", "FIELDS", ":", "uvp"]
    assert text[2].split()[:6] == ["#", "2", "NUMBER", "SETS", ":", "uv"]
    assert text[12].split()[-2:] == [str(mu.nband), str(mp.nband)]   # BANDWIDTH line
    assert len(text) == 15 + mu.nel * mu.next
    for field, m in (("v", mu), ("p", mp)):
        n = sx.read_numbering(path, field, m.nel, m.np)
        assert np.array_equal(n["btog"], m.btog) and np.array_equal(n["bmask"], m.bmask)
        assert (n["nglobal"], n["nsolve"], n["nband"]) == (m.nglobal, m.nsolve, m.nband)
    assert sx.read_numbering(path, "u", mu.nel, mu.np)["set"] == "uv"


def test_numbering_checks_like_buildnum(sx, tmp_path):
    """Mismatches of NEL / NP_MAX and a missing field are refused, as
    BCmgr::buildnum refuses them (src/bcmgr.cpp:660-750)."""
    mu, _ = _channel_pair()
    path = tmp_path / "one.num"
    sx.write_numbering(path, {"u": mu})
    with pytest.raises(sx.SolverError, match="number of elements"):
        sx.read_numbering(path, "u", mu.nel + 1, mu.np)
    with pytest.raises(sx.SolverError, match="element order"):
        sx.read_numbering(path, "u", mu.nel, mu.np + 1)
    with pytest.raises(sx.SolverError, match="no number set"):
        sx.read_numbering(path, "c", mu.nel, mu.np)


def test_numbering_with_free_spacing(sx, tmp_path):
    """The reader reads words, as the reference's stream extraction does:
    a file laid out with other column widths reads the same."""
    mu, _ = _channel_pair(renumber="none")
    path = tmp_path / "loose.num"
    rows = [f"{e + 1} {a // (mu.np - 1) + 1} {a % (mu.np - 1)} {mu.btog[e, a]} {mu.bmask[e, a]}"
            for e in range(mu.nel) for a in range(mu.next)]
    head = ["# FIELDS : u", "# --", "# 1 NUMBER SETS : u", f"# NEL : {mu.nel}", f"# NP_MAX : {mu.np}",
            f"# NEXT_MAX : {mu.next}", f"# NINT_MAX : {mu.nint}", f"# NTOTAL : {mu.nel * mu.npnp}",
            f"# NBOUNDARY : {mu.nel * mu.next}", f"# NGLOBAL : {mu.nglobal}", f"# NSOLVE : {mu.nsolve}",
            "# OPTIMIZATION : 0", f"# BANDWIDTH : {mu.nband}", "# --", "# elmt side offst bmap mask"]
    path.write_text("\n".join(head + rows) + "\n")
    n = sx.read_numbering(path, "u", mu.nel, mu.np)
    assert np.array_equal(n["btog"], mu.btog) and n["nband"] == mu.nband
