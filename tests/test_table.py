"""Table mode (-tb) argument handling on the CPU: MEGADOCK's megadock-dp table
semantics (src/mpidp.cpp:132-251, :786-878): TITLE=/PARAM= lines with the
first seven characters' spaces removed, $n substitution from tab-separated
fields, the -ot output field with the ".retry" suffix, every non-table option
passed to each job ahead of PARAM's tokens."""
import ctypes as C

import pytest


def _argv(args):
    arr = (C.c_char_p * len(args))(*[a.encode() for a in args])
    return len(args), arr


def _expand(args, job, retry=0):
    from megadock_b200 import _native as N
    n, arr = _argv(args)
    buf = C.create_string_buffer(8192)
    nj = C.c_int()
    rc = N.lib().md_table_expand(n, arr, job, retry, buf, len(buf), C.byref(nj))
    return rc, buf.value.decode().split("\n"), nj.value


def _table(tmp_path, text):
    p = tmp_path / "jobs.table"
    p.write_text(text)
    return str(p)


def test_expand_fields_and_options(built, tmp_path):
    tb = _table(tmp_path, "  TITLE=sample jobs\n PARAM=-R $1 -L $2 -o $3 -F 64\n"
                          "a_r.pdb\ta_l.pdb\ta.out\nb_r.pdb\tb_l.pdb\tb.out\n")
    args = ["megadock-b200", "-tb", tb, "-ot", "3", "-rt", "2", "-r", "24", "-lg", "x.log"]
    rc, lines, nj = _expand(args, 1)
    assert rc == 0 and nj == 2
    assert lines == ["megadock-b200", "-r", "24", "-R", "b_r.pdb", "-L", "b_l.pdb", "-o", "b.out", "-F", "64",
                     "#out b.out"]
    rc, lines, _ = _expand(args, 0, retry=2)
    assert rc == 0
    assert lines[-1] == "#out a.out.2" and "a.out.2" in lines


def test_expand_without_output_check_and_lowercase_keys(built, tmp_path):
    tb = _table(tmp_path, "title=t\nparam=-R $1 -L $2\nr.pdb\tl.pdb\n")
    rc, lines, nj = _expand(["megadock-b200", "-tb", tb], 0, retry=1)
    assert rc == 0 and nj == 1
    assert lines == ["megadock-b200", "-R", "r.pdb", "-L", "l.pdb", "#out "]


def test_table_errors(built, tmp_path):
    from megadock_b200 import _native as N
    tb = _table(tmp_path, "TITLE=no param\nr.pdb\tl.pdb\n")
    rc, _, _ = _expand(["megadock-b200", "-tb", tb], 0)
    assert rc == N.MD_ERR_USAGE
    rc, _, _ = _expand(["megadock-b200", "-tb", str(tmp_path / "missing.table")], 0)
    assert rc == N.MD_ERR_IO
    tb = _table(tmp_path, "PARAM=-R $1 -L $2\nr.pdb\tl.pdb\nshort.pdb\n")
    rc, _, nj = _expand(["megadock-b200", "-tb", tb], 1)
    assert nj == 2 and rc == N.MD_ERR_ARG
    n, arr = _argv(["megadock-b200", "-R", "x"])
    assert N.lib().md_table_mode(n, arr) == 0
    n, arr = _argv(["megadock-b200", "-tb", tb])
    assert N.lib().md_table_mode(n, arr) == 1
