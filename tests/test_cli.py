"""The museqa command line and the C++ facade (include/msa_b200.hpp): option
handling and messages as the reference's (src/museqa.cpp, src/terminal.cpp),
the C++ FASTA loader equal to the Python one on awkward files, and (on a GPU)
the whole pipeline: its distance matrix and guide tree equal the library's."""
import re
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from msa_b200 import Database, ScoringTable, pairwise, phylogeny
from msa_b200 import workloads as W

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "msa_b200" / "museqa"


def run_cli(*args, cwd=None):
    p = subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, cwd=cwd, timeout=600)
    return p.returncode, p.stdout


@pytest.mark.parametrize("args,message", [
    ((), "no input files given"),
    (("-1", "bogus", "x.fasta"), "unknown pairwise algorithm chosen: 'bogus'"),
    (("-s", "blosum1000", "x.fasta"), "unknown scoring table chosen: 'blosum1000'"),
    (("-2", "upgma", "x.fasta"), "unknown phylogeny algorithm chosen: 'upgma'"),
    (("x.fasta", "-s"), "missing argument value for option '-s'"),
])
def test_option_errors_match_the_reference(args, message):
    rc, out = run_cli(*args)
    assert rc == 1
    assert out.strip().splitlines()[-1] == f"[watchdog|error|{message}]"


def test_help():
    rc, out = run_cli("--help")
    assert rc == 0 and "--scoring-table" in out and "--pairwise" in out


FASTA_CASES = {
    "plain.fasta": b">a one\nACGT\nTTGA\n>b\nMKV\n",
    "no_newline.fa": b">x\nACDEFGHIK\n>y\nLMN",
    "crlf.fasta": b">r1\r\nACGT\r\nGG\r\n>r2\r\nTT\r\n",
    "blank_line.fasta": b">s\nACGT\n\nCCCC\n>t\nGGG\n",
    "preamble.fasta": b"junk line\n;comment\n>first\nAC-GT*x9\n>\nQ\n>empty\n>last\nwy\n",
    "empty.fasta": b"",
}


@pytest.fixture(scope="module")
def fasta_dump(tmp_path_factory):
    exe = tmp_path_factory.mktemp("bin") / "fasta_dump"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/fasta_dump.cpp"),
                    "-o", str(exe), "-L", str(ROOT / "msa_b200"), "-lmsa_b200",
                    f"-Wl,-rpath,{ROOT / 'msa_b200'}"], check=True)
    return exe


@pytest.mark.parametrize("name", sorted(FASTA_CASES))
def test_cpp_fasta_loader_equals_python(tmp_path, fasta_dump, name):
    f = tmp_path / name
    f.write_bytes(FASTA_CASES[name])
    p = subprocess.run([str(fasta_dump), str(f)], capture_output=True, timeout=60)
    assert p.returncode == 0
    got = [tuple(line.split(b"\t", 1)) for line in p.stdout.split(b"\n") if line]
    db = Database.load(str(f))
    want = [(e.description.encode("latin-1"), str(e.contents).encode()) for e in db]
    assert got == want


def _fast_path_units(files):
    import ctypes
    from msa_b200 import _lib
    lib = _lib.lib()
    arr = (ctypes.c_char_p * len(files))(*[str(f).encode() for f in files])
    ns, nu = ctypes.c_uint32(), ctypes.c_uint64()
    rc = lib.msa_fasta_count(arr, len(files), ctypes.byref(ns), ctypes.byref(nu))
    if rc:
        return rc, None
    units = np.zeros(max(nu.value, 1), np.uint8)
    offs = np.zeros(max(ns.value, 1), np.uint64)
    lens = np.zeros(max(ns.value, 1), np.uint64)
    rc = lib.msa_fasta_encode(arr, len(files), units.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                              offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                              lens.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    return rc, [units[int(o):int(o + n)] for o, n in zip(offs[:ns.value], lens[:ns.value])]


def test_fast_fasta_loader_equals_python(tmp_path):
    # The one-pass loader behind msa_seqs_load_fasta, on every awkward case
    # at once (files are merged in order, as the reference's loader does).
    files = []
    for name, data in sorted(FASTA_CASES.items()):
        f = tmp_path / name
        f.write_bytes(data)
        files.append(f)
    rc, got = _fast_path_units(files)
    assert rc == 0
    db = Database.load(*map(str, files))
    want = [e.contents.units[:e.contents.raw_length] for e in db]
    assert len(got) == len(want)
    assert all(np.array_equal(a, b) for a, b in zip(got, want))


def test_fast_fasta_loader_on_the_reference_databases():
    from oracle.oracle import REFERENCE_ROOT
    db_dir = REFERENCE_ROOT / "db"
    files = sorted(db_dir.glob("*.fasta")) if db_dir.is_dir() else []
    if not files:
        pytest.skip("the reference's FASTA databases are not present")
    for f in files[:6]:
        rc, got = _fast_path_units([f])
        assert rc == 0
        want = [e.contents.units[:e.contents.raw_length] for e in Database.load(str(f))]
        assert len(got) == len(want) and all(np.array_equal(a, b) for a, b in zip(got, want)), f.name


def test_fast_fasta_loader_errors(tmp_path):
    f = tmp_path / "x.txt"
    f.write_text(">a\nAC\n")
    assert _fast_path_units([f])[0] != 0
    assert _fast_path_units([tmp_path / "missing.fasta"])[0] != 0


def test_cpp_loader_rejects_unknown_extension(tmp_path, fasta_dump):
    f = tmp_path / "seqs.txt"
    f.write_text(">a\nAC\n")
    p = subprocess.run([str(fasta_dump), str(f)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1 and "unknown database parser 'txt'" in p.stdout


def _newick_parts(text):
    """Structure with the numbers taken out, and the numbers as float32."""
    nums = re.findall(r":([^,();]+)", text)
    return re.sub(r":[^,();]+", ":", text.strip()), np.array([float(x) for x in nums], np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("extra", [[], ["-m"], ["-1", "sequential", "-2", "njoining-sequential"]])
def test_pipeline_matches_the_library(gpu, tmp_path, extra):
    wl = W.random_set(31, 40, 50, 400)
    fasta = tmp_path / "seqs.fasta"
    fasta.write_bytes(b"".join(b">s%d\n%s\n" % (k, bytes(s)) for k, s in enumerate(wl.seqs)))
    rc, out = run_cli("-s", "blosum62", *extra, "--newick", tmp_path / "tree.nwk", "--matrix", tmp_path / "m.bin",
                      fasta)
    assert rc == 0, out
    lines = out.splitlines()
    assert "[watchdog|info|loaded a total of <bold>40</> sequences]" in lines
    assert "[watchdog|init|pairwise|aligning <bold>780</> pairs]" in lines
    assert "[watchdog|finish|phylogeny|phylogenetic tree produced]" in lines
    for task in ("loading", "pairwise", "phylogeny", "total"):
        assert any(re.fullmatch(rf"\[watchdog\|report\|{task}\|\d+\.\d{{6}}\]", ln) for ln in lines), task

    raw = (tmp_path / "m.bin").read_bytes()
    assert raw[:4] == b"MSAT" and struct.unpack("<I", raw[4:8])[0] == 40
    tri = np.frombuffer(raw[8:], np.int32)
    db = Database.load(str(fasta))
    want = pairwise.run(db, ScoringTable("blosum62"))
    assert np.array_equal(tri, want.int_scores)

    tree = phylogeny.run(want)
    s_cli, d_cli = _newick_parts((tmp_path / "tree.nwk").read_text())
    s_py, d_py = _newick_parts(tree.newick([e.description for e in db]))
    assert s_cli == s_py
    # Same float bits, NaN (the last join's 0/0 branch lengths) matched as NaN:
    # text NaN keeps no payload and Python's repr drops its sign.
    nan = np.isnan(d_cli)
    assert np.array_equal(nan, np.isnan(d_py))
    assert np.array_equal(d_cli[~nan].view(np.uint32), d_py[~nan].view(np.uint32))


@pytest.mark.gpu
def test_report_only_prints_only_reports(gpu, tmp_path):
    fasta = tmp_path / "s.fa"
    fasta.write_text(">a\nMKVLA\n>b\nMKVIA\n>c\nMRVLA\n")
    rc, out = run_cli("-r", fasta)
    assert rc == 0
    events = {ln.split("|")[1] for ln in out.splitlines()}
    assert events <= {"report", "warning"}


@pytest.mark.gpu
def test_fasta_straight_to_device_store(gpu, tmp_path):
    import ctypes
    from msa_b200 import _lib, runtime
    wl = W.random_set(32, 30, 20, 300)
    fasta = tmp_path / "s.fasta"
    fasta.write_bytes(b"".join(b">seq %d\r\n%s\n" % (k, bytes(s)) for k, s in enumerate(wl.seqs)))
    ctx = runtime.context(0)
    lib = _lib.lib()
    arr = (ctypes.c_char_p * 1)(str(fasta).encode())
    h, n = ctypes.c_uint64(), ctypes.c_uint32()
    _lib.check(lib.msa_seqs_load_fasta(ctx.handle, arr, 1, ctypes.byref(h), ctypes.byref(n)), ctx.handle)
    try:
        db = Database.load(str(fasta))
        assert n.value == db.count
        assert [lib.msa_seqs_description(ctx.handle, h.value, k).decode("latin-1") for k in range(n.value)] == \
               [e.description for e in db]
        out = np.zeros(n.value * (n.value - 1) // 2, np.int32)
        t = ScoringTable("blosum62")
        _lib.check(lib.msa_nw_all_pairs(ctx.handle, h.value, ctypes.byref(t._t), _lib.MSA_NW_PERSISTENT,
                                        out.ctypes.data_as(ctypes.c_void_p), 0), ctx.handle)
        assert np.array_equal(out, pairwise.run(db, t).int_scores)
    finally:
        lib.msa_seqs_release(ctx.handle, h.value)
